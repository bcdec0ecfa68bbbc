"""The optional two-level Poisson preconditioner (``coarse_box_nodes > 0``) on the GPU.

No counterpart in the reference, whose Poisson PCG (``scripts/solvers.py:221-231``) is
preconditioned by the diagonal.  The two-level form adds a coarse correction on spatial
boxes of nodes, ``z = r/diag + P Ac^-1 P^T r``; the stop test stays the reference's
``r.r <= tol_u^2 b.b``, so energies and gradients must agree with the oracle's Jacobi solve
as closely as two solves to that tolerance agree (1e-9 relative in FP64; mixed precision adds
the FP32 rounding of the operator values, tests/test_gpu_mixed.py), while the iteration
count follows the oracle's two-level PCG on the same boxes.
"""

import numpy as np
import pytest

import oracle as O
from mammos_mumag import _native, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grains():
    return synthetic.multigrain(n=12, L=30.0, grains=3, cone_deg=20.0, gb=2.0, seed=3)


@pytest.mark.parametrize("precision", [_native.PREC_FP64, _native.PREC_MIXED])
def test_coarse_energy_gradient_match_oracle(grains, precision):
    X, T, tag, krn, m0 = grains
    P = O.Problem(X, T, tag, krn)
    hdir = [0.0, 0.0, 1.0]
    with _native.Mesh(X, T, tag, krn, precision=precision, coarse_box_nodes=64) as M:
        box, nb = M.coarse()
        assert nb > 8 and M.info()["coarse_boxes"] == nb
        assert np.all(box[P.bnd] == -1) and np.all(box[~P.bnd] >= 0)
        M.set_state(m0, None, m0)
        E, gp, it = M.energy_grad(0.4, _native.solver_params(hdir=hdir))
        _, u, _ = M.get_state()
    Eo, gpo, uo, _ = O.total_eg(P, m0, 0.4, hdir, np.zeros(P.N), 1e-10)
    assert E == pytest.approx(Eo, rel=1e-9 if precision == _native.PREC_FP64 else 2e-7)
    assert np.abs(gp - gpo).max() <= 1e-7 * np.abs(gpo).max()
    assert np.abs(u - uo).max() <= 1e-7 * np.abs(uo).max()
    b = P.divergence(m0)
    _, kj = O.pcg(P.S, P.diagS, b, np.zeros(P.N), 1e-10)
    _, kc = O.pcg_twolevel(P.S, P.diagS, b, np.zeros(P.N), 1e-10, box)
    assert kc < kj
    if precision == _native.PREC_FP64:
        # the same iteration in another arrangement: the count agrees up to rounding at the stop
        assert abs(it - kc) <= 1, (it, kc, kj)
    else:
        # FP32 inner solves to 1e-5 restarted by FP64 refinement: a few more
        assert kc <= it <= 2 * kc + 10, (it, kc, kj)


def test_coarse_field_step_matches_jacobi(grains):
    """One field step (the reference's NCG with every evaluation's Poisson solve) with the
    two-level preconditioner ends where the Jacobi path ends, within the loop tolerance of
    the NCG stopping rule, and takes fewer PCG iterations."""
    X, T, tag, krn, m0 = grains
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    res = {}
    for cb in (0, 64):
        with _native.Mesh(X, T, tag, krn, coarse_box_nodes=cb) as M:
            M.set_state(m0, None, m0)
            res[cb] = M.minimize(-1.0, sp)
    a, b = res[0], res[64]
    assert a["status"] == 0 and b["status"] == 0
    assert b["energy"] == pytest.approx(a["energy"], rel=1e-6)
    assert b["mh"] == pytest.approx(a["mh"], rel=1e-4)
    assert b["pcg_iters"] / b["evals"] < a["pcg_iters"] / a["evals"]


def test_coarse_launch_shapes_and_staging_agree(grains):
    """The box sums follow the CTA partition, so other grids round differently: energies agree
    to 1e-10; staged and streamed operators give identical results on one grid."""
    X, T, tag, krn, m0 = grains
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    out = []
    for grid, stage in ((0, 1), (0, 0), (37, 1), (5, 1)):
        with _native.Mesh(X, T, tag, krn, coarse_box_nodes=64, grid_ctas=grid, stage_operators=stage) as M:
            M.set_state(m0, None, m0)
            E, gp, it = M.energy_grad(0.3, sp)
            out.append((E, gp, it))
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])
    for E, gp, it in out[2:]:
        assert E == pytest.approx(out[0][0], rel=1e-10)
        assert abs(it - out[0][2]) <= 1


def test_coarse_with_learned_start(grains):
    """The learned warm start feeds the two-level solve: the start changes, the solution
    criterion does not."""
    X, T, tag, krn, m0 = grains
    P = O.Problem(X, T, tag, krn)
    hdir = [0.0, 0.0, 1.0]
    with _native.Model(seed=5) as net, _native.Mesh(X, T, tag, krn, precision=_native.PREC_MIXED,
                                                    coarse_box_nodes=64) as M:
        M.set_warm_start(_native.WARM_LEARNED, net)
        M.set_state(m0, None, m0)
        E, gp, it = M.energy_grad(0.4, _native.solver_params(hdir=hdir))
    Eo, gpo, _, _ = O.total_eg(P, m0, 0.4, hdir, np.zeros(P.N), 1e-10)
    assert E == pytest.approx(Eo, rel=2e-7)  # mixed precision (tests/test_gpu_mixed.py)
    assert np.abs(gp - gpo).max() <= 1e-7 * np.abs(gpo).max()


def test_coarse_on_shell_mesh(cube_mesh, golden):
    """The reference's cube in its spherical shell (the boundary branch its goldens pin):
    the two-level solve gives the magnetostatic energy the Jacobi solve gives (which
    tests/test_gpu_parity.py holds to the reference's tests/data/hmag known answer)."""
    X, T, tag = cube_mesh
    krn = O.read_krn_rows((golden / "loop_cube.krn").read_text())
    P = O.Problem(X, T, tag, krn)
    mu = O.initial_m_uniform(P, [0.0, 0.0, 1.0])
    on, off = _native.solver_params(hmag_on=1), _native.solver_params(hmag_on=0)
    res = {}
    for cb in (0, 128):
        with _native.Mesh(X, T, tag, krn, coarse_box_nodes=cb) as M:
            M.set_state(mu, None, mu)
            e_on, _, it = M.energy_grad(0.0, on)
            M.set_state(mu, None, mu)
            e_off, _, _ = M.energy_grad(0.0, off)
            res[cb] = ((e_on - e_off) / O.MU0_OUT, it)
    assert res[128][0] == pytest.approx(res[0][0], rel=1e-9)
    assert res[128][1] < res[0][1]
