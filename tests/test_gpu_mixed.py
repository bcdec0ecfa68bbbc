"""Mixed precision (MM_PREC_MIXED): FP32 copies of every operator plane (Poisson, exchange,
anisotropy, divergence, gradient) read with FP64 vectors and FP64 sums, FP32 inner PCG
iterations, FP64 residual refinement, reductions and stop tests; M_inv's truncated CG keeps
its vectors (r, z, d, B d) in FP32 with FP64 arithmetic and sums.

Bars: energies and fields of one evaluation within the FP32 rounding of the operator values
(the FP32 planes define a slightly perturbed but consistent energy: 2-4e-8 relative on these
meshes, checked with the oracle's operators rounded the same way; 2e-7 is the bound used
here, inside the contract's 1e-6 for FP64 mode); loop coercivity Hc and remanence Mr within
1 % of the FP64 path."""

import numpy as np
import pytest

import oracle as O
from mammos_mumag import _native, synthetic
from mammos_mumag.hysteresis import coercivity_remanence as hc_mr

pytestmark = pytest.mark.gpu




@pytest.fixture(scope="module")
def grains():
    return synthetic.multigrain(n=8, L=20.0, grains=3, cone_deg=20.0, gb=2.0, seed=7)


def test_mixed_energy_gradient_matches_oracle(grains):
    X, T, tag, krn, m0 = grains
    P = O.Problem(X, T, tag, krn)
    hdir = [0.0, 0.0, 1.0]
    with _native.Mesh(X, T, tag, krn, precision=_native.PREC_MIXED) as M:
        M.set_state(m0, None, m0)
        E, gp, it = M.energy_grad(0.4, _native.solver_params(hdir=hdir))
        _, u, _ = M.get_state()
    Eo, gpo, uo, _ = O.total_eg(P, m0, 0.4, hdir, np.zeros(P.N), 1e-10)
    assert E == pytest.approx(Eo, rel=2e-7)
    assert np.abs(gp - gpo).max() <= 1e-7 * np.abs(gpo).max()
    assert np.abs(u - uo).max() <= 1e-7 * np.abs(uo).max()
    assert it > 0


def test_mixed_minv_close_to_fp64(grains):
    X, T, tag, krn, m0 = grains
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    out = {}
    for prec in (_native.PREC_FP64, _native.PREC_MIXED):
        with _native.Mesh(X, T, tag, krn, precision=prec) as M:
            M.set_state(m0, None, m0)
            M.energy_grad(0.4, sp)
            _, _, gf = M.get_state()
            g = O.projection(m0, gf)
            out[prec], _ = M.apply_minv(g, sp)
    z64, z32 = out[_native.PREC_FP64], out[_native.PREC_MIXED]
    assert np.abs(z32 - z64).max() <= 1e-4 * np.abs(z64).max()


def test_mixed_loop_hc_mr_within_one_percent(grains):
    X, T, tag, krn, m0 = grains
    d = np.radians(1.0)
    hdir = [np.sin(d), 0.0, np.cos(d)]
    res = {}
    for prec in (_native.PREC_FP64, _native.PREC_MIXED):
        with _native.Mesh(X, T, tag, krn, precision=prec) as M:
            M.set_state(m0, None, m0)
            rows, steps = M.loop(2.0, -6.0, -0.25, 0.4, -2.0, _native.solver_params(hdir=hdir))
            res[prec] = (rows, steps)
    r64, r32 = res[_native.PREC_FP64][0], res[_native.PREC_MIXED][0]
    assert r64.shape == r32.shape
    hc64, mr64 = hc_mr(r64)
    hc32, mr32 = hc_mr(r32)
    assert np.isfinite(hc64) and np.isfinite(mr64), "the sweep must switch"
    assert abs(hc32 - hc64) <= 0.01 * hc64
    assert abs(mr32 - mr64) <= 0.01 * abs(mr64)
    np.testing.assert_allclose(r32[:, 3], r64[:, 3], rtol=1e-4)
