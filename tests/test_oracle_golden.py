"""Pin the CPU oracle against the reference's own recorded outputs (tests/golden)."""

import pathlib

import numpy as np
import pytest

import oracle as O

ROOT = pathlib.Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def cube_problem(cube_mesh, golden):
    X, T, tag = cube_mesh
    krn = O.read_krn_rows((golden / "loop_cube.krn").read_text())
    return O.Problem(X, T, tag, krn)


def test_shell_branch_detected(cube_problem):
    P = cube_problem
    assert not P.airbox
    assert P.V == pytest.approx(8000.0, rel=1e-12)
    assert P.bnd.sum() > 8


def test_loop_matches_cube_dat(cube_problem, golden):
    """The whole loop (tests/data/loop/cube.dat, 21 rows, tests/test_loop.py:21-23)."""
    par = O.read_params((golden / "loop_cube.p2").read_text())
    snaps = {}
    rows, st = O.run_loop(
        cube_problem, par, snapshot=lambda c, m, u: snaps.setdefault(c, (m.copy(), u.copy()))
    )
    gold = np.loadtxt(golden / "loop_cube.dat")
    out = rows.copy()
    out[:, 3] /= O.MU0_OUT
    assert out.shape == gold.shape
    assert np.array_equal(out[:, 0], gold[:, 0])
    assert np.array_equal(out[:, 1], gold[:, 1])  # cumulative float field values, bit-exact
    np.testing.assert_allclose(out[:, 2], gold[:, 2], rtol=1e-12)
    np.testing.assert_allclose(out[:, 3], gold[:, 3], rtol=1e-12)
    # the work of this loop in the reference's algorithm: 67 NCG iterations, 113 evaluations
    assert sum(s.ncg_iters for s in st) == 67
    assert sum(s.evals for s in st) == 113
    # the written .dat rows parse to the golden values
    text = O.format_dat(rows)
    np.testing.assert_allclose(np.loadtxt(text.splitlines()), gold, rtol=1e-12)
    # the snapshot tests/data/loop/cube_0001.vtu (ASCII, 7 significant digits)
    v = np.load(golden / "loop_cube_0001.npz")
    m1, u1 = snaps[1]
    assert list(snaps) == [1]
    np.testing.assert_allclose(m1.reshape(-1, 3), v["m"], rtol=1e-5, atol=2e-7)
    np.testing.assert_allclose(u1, v["u"], rtol=1e-5, atol=2e-6)


def test_hmag_energy(cube_problem, energies):
    """tests/data/hmag/cube.csv E_gradient (uniform +z, shell transformation)."""
    P = cube_problem
    m = O.initial_m_uniform(P, [0.0, 0.0, 1.0])
    u, _ = O.pcg(P.S, P.diagS, P.divergence(m), np.zeros(P.N), 1e-10)
    gh = np.stack([P.gk[c] @ u for c in range(3)], 1).ravel()
    assert 0.5 * m @ gh / O.MU0_OUT == pytest.approx(energies["hmag"]["E_gradient"], rel=1e-11)


def test_exchange_anisotropy_energies(cube_problem, energies):
    P = cube_problem
    mv, _ = O.vortex_m(P)
    assert 0.5 * mv @ (P.C @ mv) / O.MU0_OUT == pytest.approx(
        energies["exani_vortex"]["E_gradient"], rel=1e-12
    )
    m = O.initial_m_uniform(P, [0.0, 0.0, 1.0])
    assert 0.5 * m @ (P.C @ m) / O.MU0_OUT == pytest.approx(
        energies["exani_uniform"]["E_gradient"], rel=1e-12
    )


def test_zeeman_energy(cube_problem, energies):
    P = cube_problem
    par = O.read_params(energies["p2"]["external"])
    h = par["hstart"] - par["hstep"]  # scripts/external.py:105
    m = O.initial_m_uniform(P, par["m"])
    e = m @ O.external_g(P, h, par["hdir"]) / O.MU0_OUT
    assert e == pytest.approx(energies["external"]["E_gradient"], rel=1e-12)


def test_mapping_float32_energies(cube_problem, energies):
    """tests/data/mapping/*.csv were written by float32 JAX: compare at the reference's
    own tolerance (np.allclose, tests/test_mapping.py)."""
    P = cube_problem
    par = O.read_params(energies["p2"]["mapping"])
    m = O.initial_m_uniform(P, par["m"])
    h = par["hstart"] - par["hstep"]
    mp = energies["mapping"]
    E, _, _, _ = O.total_eg(P, m, h, par["hdir"], np.zeros(P.N), par["tol_u"])
    assert np.allclose(E / O.MU0_OUT, mp["energy"]["E_jax"])
    assert np.allclose(m @ O.external_g(P, h, par["hdir"]) / O.MU0_OUT, mp["zeeman"]["E_jax"])
    assert np.allclose(0.5 * m @ (P.C @ m) / O.MU0_OUT, mp["anisotropy"]["E_jax"])
    mv, _ = O.vortex_m(P)
    assert np.allclose(0.5 * mv @ (P.C @ mv) / O.MU0_OUT, mp["exchange"]["E_jax"])


def test_pcg_matches_dense_solve():
    """The restated jax CG converges to the direct solution on a small SPD system."""
    rng = np.random.default_rng(0)
    A = rng.standard_normal((40, 40))
    A = A @ A.T + 40 * np.eye(40)
    b = rng.standard_normal(40)
    x, k = O.pcg(A, np.diag(A).copy(), b, np.zeros(40), 1e-12)
    np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=1e-9)
    assert 0 < k < 40


def test_twolevel_pcg_meets_the_same_stop_rule_in_fewer_iterations():
    """The oracle's two-level PCG (the checker of the GPU's box-aggregate preconditioner)
    solves the reference's Poisson system of a multigrain mesh to the reference's stop rule
    r.r <= tol^2 b.b, agrees with the Jacobi solve to that accuracy, and needs fewer
    iterations; one box holding every interior node is also a valid aggregate."""
    from mammos_mumag import synthetic

    X, T, tag, krn, m0 = synthetic.multigrain(n=12, L=30.0, grains=4, cone_deg=15.0, gb=2.0, seed=3)
    P = O.Problem(X, T, tag, krn)
    b = P.divergence(m0)
    x0 = np.zeros(P.N)
    xj, kj = O.pcg(P.S, P.diagS, b, x0, 1e-10)
    nb = 4  # 4^3 geometric boxes over the interior nodes, Dirichlet nodes in none
    lo, hi = P.X.min(0), P.X.max(0)
    ijk = np.minimum(((P.X - lo) / (hi - lo) * nb).astype(int), nb - 1)
    box = ijk[:, 0] + nb * (ijk[:, 1] + nb * ijk[:, 2])
    box[P.bnd] = -1
    inner = box >= 0
    box[inner] = np.unique(box[inner], return_inverse=True)[1].ravel()  # no empty boxes
    for agg in (box, np.where(P.bnd, -1, 0)):
        xc, kc = O.pcg_twolevel(P.S, P.diagS, b, x0, 1e-10, agg)
        r = b - P.S @ xc
        assert r @ r <= 1e-20 * (b @ b)
        assert np.abs(xc - xj).max() <= 1e-7 * np.abs(xj).max()
        assert 0 < kc < kj


def test_single_grain_sweep_fixture_is_the_oracles():
    """tests/golden/sweep_single.npz (the single-grain sweep through switching that the GPU
    sweeps are compared with) is what the oracle computes: regenerated here (a few seconds)."""
    import json
    import sys

    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_sweeps
    from mammos_mumag.hysteresis import coercivity_remanence

    f = np.load(ROOT / "tests" / "golden" / "sweep_single.npz")
    assert json.loads(str(f["params"])) == make_sweeps.CASES["single"]
    X, T, tag, krn, m0, par = make_sweeps.build_case("single")
    rows, stats = O.run_loop(O.Problem(X, T, tag, krn), par, m0=m0)
    # the BLAS thread count changes the summation order of the dense dot products: rows
    # agree to a few 1e-10, far inside the loop tolerance
    np.testing.assert_array_equal(rows[:, :2], f["rows"][:, :2])
    np.testing.assert_allclose(rows[:, 2:], f["rows"][:, 2:], rtol=1e-8, atol=1e-10)
    hc, mr = coercivity_remanence(rows)
    assert hc == pytest.approx(float(f["hc"]), rel=1e-8)
    assert mr == pytest.approx(float(f["mr"]), rel=1e-8)
    # the sweep crosses the coercive field: a switched, saturated end state
    assert rows[0, 2] > 1.5 and rows[-1, 2] < -1.5
