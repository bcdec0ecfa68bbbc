"""The two arrangements of the Poisson PCG iteration (one grid synchronisation per
iteration with neighbour z recomputed from gathered records, or two with z stored and
gathered alone) compute the same iterates: same iteration counts, same potentials and
energies (the partial sums are accumulated in the same order, so they agree to the bit
in practice; the bound below allows for a different FMA contraction)."""

import numpy as np
import pytest

from mammos_mumag import _native, synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_native.PREC_FP64, _native.PREC_MIXED])
@pytest.mark.parametrize("ctas_per_sm", [2, 3])
def test_pcg_arrangements_agree(precision, ctas_per_sm):
    X, T, tag, krn, m0 = synthetic.multigrain(n=12, L=20.0, grains=3, cone_deg=20.0, gb=2.0, seed=11)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    out = {}
    for variant in (1, 2):
        with _native.Mesh(X, T, tag, krn, precision=precision, pcg_variant=variant, ctas_per_sm=ctas_per_sm,
                          grid_ctas=24) as M:
            assert M.info()["pcg_variant"] == variant and M.info()["kernel_ctas_per_sm"] == ctas_per_sm
            M.set_state(m0, None, m0)
            E, g, it = M.energy_grad(0.5, sp)
            r1 = M.minimize(-1.0, sp)
            m, u, _ = M.get_state()
            out[variant] = (E, g, it, r1, m, u)
    a, b = out[1], out[2]
    assert a[2] == b[2] and a[3]["pcg_iters"] == b[3]["pcg_iters"] and a[3]["evals"] == b[3]["evals"]
    assert a[0] == pytest.approx(b[0], rel=1e-13)
    assert np.abs(a[1] - b[1]).max() <= 1e-12 * np.abs(a[1]).max()
    assert np.abs(a[5] - b[5]).max() <= 1e-12 * np.abs(a[5]).max()
    assert a[3]["energy"] == pytest.approx(b[3]["energy"], rel=1e-12)


def test_kernel_builds_agree():
    """The two- and three-CTA-per-SM builds of the persistent kernel, on the same launch
    shape, give the same field step."""
    X, T, tag, krn, m0 = synthetic.multigrain(n=12, L=20.0, grains=3, cone_deg=20.0, gb=2.0, seed=13)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    res = {}
    for mb in (2, 3):
        with _native.Mesh(X, T, tag, krn, ctas_per_sm=mb, grid_ctas=30) as M:
            M.set_state(m0, None, m0)
            r = M.minimize(-1.0, sp)
            res[mb] = (r, M.get_state()[0])
    (ra, ma), (rb, mb_) = res[2], res[3]
    assert ra["pcg_iters"] == rb["pcg_iters"] and ra["ncg_iters"] == rb["ncg_iters"]
    assert ra["energy"] == pytest.approx(rb["energy"], rel=1e-12)
    assert np.abs(ma - mb_).max() < 1e-10


def test_autotune_reports_a_variant():
    X, T, tag, krn, m0 = synthetic.multigrain(n=10, L=15.0, grains=2, cone_deg=20.0, gb=2.0, seed=12)
    with _native.Mesh(X, T, tag, krn) as M:
        M.set_state(m0, None, m0)
        M.autotune(_native.solver_params(hdir=[0.0, 0.0, 1.0]))
        assert M.info()["pcg_variant"] in (1, 2) and M.info()["kernel_ctas_per_sm"] in (2, 3)


@pytest.mark.parametrize("precision", [_native.PREC_FP64, _native.PREC_MIXED])
@pytest.mark.parametrize("variant", [1, 2])
def test_streamed_operators_match_staged(precision, variant):
    """Operators read from HBM (the path of meshes too large for shared memory) give the
    field step of operators staged in shared memory: same data, same arithmetic order, so
    the same numbers.  Four CTAs, so that every warp walks several slices."""
    X, T, tag, krn, m0 = synthetic.multigrain(n=12, L=20.0, grains=3, cone_deg=20.0, gb=2.0, seed=14)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    res = {}
    for stage in (1, 0):
        with _native.Mesh(X, T, tag, krn, precision=precision, pcg_variant=variant, ctas_per_sm=3, grid_ctas=4,
                          stage_operators=stage) as M:
            assert M.info()["staged"] == stage
            M.set_state(m0, None, m0)
            E, g, it = M.energy_grad(0.5, sp)
            r = M.minimize(-1.0, sp)
            m, u, _ = M.get_state()
            res[stage] = (E, g, it, r, m, u)
    a, b = res[1], res[0]
    assert a[2] == b[2] and a[3]["pcg_iters"] == b[3]["pcg_iters"] and a[3]["evals"] == b[3]["evals"]
    assert a[0] == pytest.approx(b[0], rel=1e-14)
    assert np.abs(a[1] - b[1]).max() <= 1e-13 * np.abs(a[1]).max()
    assert a[3]["energy"] == pytest.approx(b[3]["energy"], rel=1e-14)
    assert np.abs(a[4] - b[4]).max() <= 1e-13
    assert np.abs(a[5] - b[5]).max() <= 1e-13 * np.abs(a[5]).max()
