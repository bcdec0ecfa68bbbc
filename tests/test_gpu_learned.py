"""Learned warm start: the network kernels against the NumPy oracle (forward, gradients,
training), the in-kernel features and targets against the oracle on a mesh, and the warm
start's effect on PCG iterations against the reference's previous-u start and a zero start.

Tolerances: the kernels round the normalised input, the hidden weights and activations to
BF16 (8-bit significand, relative rounding 2^-9) and accumulate in FP32; the oracle rounds
at the same points and accumulates in float64, so outputs agree to a few BF16 ulps of the
activations.  The kernels' backward pass also rounds the back-propagated errors to BF16, so
gradients agree with the oracle's exact gradient to about a percent."""

import numpy as np
import pytest

import oracle as O
from oracle import mlp_oracle as MO
from mammos_mumag import _native, learned, synthetic

pytestmark = pytest.mark.gpu


def _model_and_data(seed=0, n=256):
    rng = np.random.default_rng(seed)
    model = _native.Model(seed=seed)
    feats = rng.standard_normal((n, 16)).astype(np.float32) * 2 + 0.5
    target = (np.tanh(feats[:, 0] * feats[:, 3]) + 0.3 * feats[:, 12]).astype(np.float32)
    model.fit_normalization(feats, target)
    return model, feats, target


@pytest.mark.parametrize("rows", [512, 1000, 20000])
def test_predict_matches_oracle(rows):
    """mm_model_predict runs the tcgen05 kernel: 128-row tiles, the last one partial."""
    model, feats, _ = _model_and_data(1, rows)
    p = model.get_params()
    fm, fs, osc = model.get_normalization()
    y = model.predict(feats)
    yo, _ = MO.forward(p, fm, fs, feats)
    yo = yo * osc
    assert np.abs(y - yo).max() <= 2e-2 * np.sqrt(np.mean(yo ** 2)) + 1e-6


def test_gradient_matches_oracle():
    model, feats, target = _model_and_data(2, 256)
    p = model.get_params()
    fm, fs, osc = model.get_normalization()
    # move the head away from its small initialisation so every layer gets a gradient
    P = MO.unpack(p)
    P["w4"] = np.random.default_rng(3).standard_normal(128) * 0.2
    p = MO.pack(P).astype(np.float32)
    model.set_params(p)
    loss, g = model.grad(feats, target)
    yo, cache = MO.forward(p, fm, fs, feats)
    lo = MO.loss(yo, target, osc)
    go = MO.backward(p.astype(np.float64), cache, yo, target, osc)
    assert loss == pytest.approx(lo, rel=1e-2)
    G, Go = MO.unpack(g), MO.unpack(go)
    for name in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4"):
        a, b = G[name].ravel(), Go[name].ravel()
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert err < 3e-2 and cos > 0.999, (name, err, cos)


def test_training_reduces_loss():
    model, feats, target = _model_and_data(4, 4096)
    l0, _ = model.grad(feats, target)
    l1 = model.train(feats, target, epochs=20, batch=256, lr=2e-3, seed=1)
    l2, _ = model.grad(feats, target)
    assert np.isfinite(l1) and l2 < 0.2 * l0


def test_recorded_features_and_targets_match_oracle():
    X, T, tag, krn, m0 = synthetic.multigrain(n=6, L=15.0, grains=2, cone_deg=20.0, gb=2.0, seed=3)
    P = O.Problem(X, T, tag, krn)
    rng = np.random.default_rng(5)
    u_prev = rng.standard_normal(P.N) * 0.1
    m = m0.reshape(-1, 3) + 0.2 * rng.standard_normal((P.N, 3))
    m = (m / np.linalg.norm(m, axis=1, keepdims=True)).ravel()
    hdir = [0.0, 0.0, 1.0]
    with _native.Mesh(X, T, tag, krn) as M:
        M.set_state(m, u_prev, m)
        M.record_samples(2 * P.N, stride=1, seed=1)
        M.energy_grad(0.3, _native.solver_params(hdir=hdir))
        f, t, node = M.read_samples()
        _, u_new, _ = M.get_state()
    assert len(node) == P.N and np.array_equal(np.sort(node), np.arange(P.N))
    b = P.divergence(m)
    r0 = b - P.S @ u_prev
    F, sig = MO.node_features(MO.node_graph(T, P.N), m, u_prev, r0, P.diagS)
    Fo = F[node]
    scale = np.maximum(np.abs(Fo).max(axis=0), 1e-30)
    assert (np.abs(f - Fo) / scale).max() < 1e-5
    to = (u_new - u_prev)[node] / sig
    assert np.abs(t - to).max() <= 1e-5 * np.abs(to).max()


@pytest.fixture(scope="module")
def small_experiment():
    spec = learned.LoopSpec(n=10, L=15.0, grains=3, hstep=-0.4)
    feats, targets = learned.collect(range(8), spec, samples=16000)
    model, loss = learned.train(feats, targets, epochs=15)
    res = learned.compare(model, [200, 201], spec)
    return spec, model, loss, res


def test_learned_start_keeps_loop_results(small_experiment):
    _, _, loss, res = small_experiment
    assert loss < 1.0
    for a, b in zip(res["previous"]["per_seed"], res["learned"]["per_seed"]):
        ra, rb = a["rows"], b["rows"]
        n = min(len(ra), len(rb))
        assert np.abs(ra[:n, 2] - rb[:n, 2]).max() < 1e-3
        hca, hcb = a["hc_mr"][0], b["hc_mr"][0]
        if np.isfinite(hca):
            assert abs(hca - hcb) <= 0.01 * hca


def test_learned_start_fewer_pcg_iterations(small_experiment):
    _, _, _, res = small_experiment
    prev, zero, lrn = (res[k]["pcg_per_solve"] for k in ("previous", "zero", "learned"))
    print(f"PCG iterations per solve: previous-u {prev:.2f}, zero {zero:.2f}, learned {lrn:.2f}")
    assert prev < zero
    assert lrn < prev


def test_learned_start_tensor_core_path_matches_mma_sync_path():
    """The learned start runs its network on tcgen05 when the launch has at most one CTA per
    SM (100 CTAs here) and on mma.sync otherwise (200 CTAs of the three-CTA-per-SM build):
    same solve, the warm start differing only by the network's rounding."""
    X, T, tag, krn, m0 = synthetic.multigrain(n=20, L=25.0, grains=3, cone_deg=20.0, gb=2.0, seed=9)
    rng = np.random.default_rng(3)
    feats = rng.standard_normal((4096, 16)).astype(np.float32)
    model, _ = learned.train(feats, (0.1 * feats[:, 12]).astype(np.float32), epochs=2)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    m1 = m0.reshape(-1, 3) + 0.05 * rng.standard_normal((len(m0) // 3, 3))
    m1 = (m1 / np.linalg.norm(m1, axis=1, keepdims=True)).ravel()
    out = {}
    for grid, mb in ((100, 2), (200, 3)):
        with _native.Mesh(X, T, tag, krn, grid_ctas=grid, ctas_per_sm=mb) as M:
            assert M.info()["grid_ctas"] == grid
            M.set_warm_start(_native.WARM_LEARNED, model)
            M.set_state(m0, None, m0)
            M.energy_grad(0.3, sp)
            M.set_state(m1, M.get_state()[1], m0)
            E, g, it = M.energy_grad(0.3, sp)
            out[grid] = (E, M.get_state()[1], it)
    (Ea, ua, ia), (Eb, ub, ib) = out[100], out[200]
    assert abs(ia - ib) <= 2
    assert np.abs(ua - ub).max() <= 1e-8 * np.abs(ua).max()
    assert Ea == pytest.approx(Eb, rel=1e-10)
    model.close()
