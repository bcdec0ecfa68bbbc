"""The network oracle itself (CPU): its backward pass against finite differences, and its
BF16 rounding against torch's bfloat16 conversion."""

import numpy as np
import torch

from oracle import mlp_oracle as MO


def _params(rng, scale=1.0):
    p = rng.standard_normal(MO.num_params()) * 0.1 * scale
    return p


def test_param_count_matches_layout():
    assert MO.num_params() == 16 * 128 + 128 + 2 * (128 * 128 + 128) + 128 + 1


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(rng)
    F = rng.standard_normal((32, 16))
    t = rng.standard_normal(32)
    fm, fs, osc = np.zeros(16), np.ones(16), 1.7
    y, cache = MO.forward(p, fm, fs, F, quantize=False)
    g = MO.backward(p, cache, y, t, osc)
    idx = rng.choice(p.size, 60, replace=False)
    idx = np.concatenate([idx, [p.size - 1, p.size - 2]])  # b4 and the last w4 entry
    eps = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += eps
        pm[k] -= eps
        lp = MO.loss(MO.forward(pp, fm, fs, F, quantize=False)[0], t, osc)
        lm = MO.loss(MO.forward(pm, fm, fs, F, quantize=False)[0], t, osc)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (k, fd, g[k])


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(10000) * 10 ** rng.uniform(-8, 8, 10000), [0.0, -0.0, 1.0, 65504.0]])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(MO.bf16(x), ref)


def test_node_features_small_mesh():
    # two tets sharing a face: nodes 0..4
    T = np.array([[0, 1, 2, 3], [1, 2, 3, 4]])
    G = MO.node_graph(T, 5)
    m = np.arange(15, dtype=float) / 15.0
    u = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    r0 = np.array([1.0, -1.0, 2.0, 0.5, 0.0])
    diag = np.full(5, 2.0)
    F, sig = MO.node_features(G, m, u, r0, diag)
    z = r0 / diag
    assert np.isclose(sig, np.sqrt(np.mean(z * z)))
    # node 0 sees nodes 0..3, node 4 sees 1..4
    assert np.isclose(F[0, 7], np.mean(u[:4])) and np.isclose(F[4, 7], np.mean(u[1:]))
    assert np.isclose(F[0, 11], 4.0) and np.isclose(F[4, 11], 5.0)
    assert np.isclose(F[4, 15], z[1:].min() / sig) and np.isclose(F[0, 14], z[:4].max() / sig)
