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
def test_pcg_arrangements_agree(precision):
    X, T, tag, krn, m0 = synthetic.multigrain(n=12, L=20.0, grains=3, cone_deg=20.0, gb=2.0, seed=11)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    out = {}
    for variant in (1, 2):
        with _native.Mesh(X, T, tag, krn, precision=precision, pcg_variant=variant) as M:
            assert M.info()["pcg_variant"] == variant
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


def test_autotune_reports_a_variant():
    X, T, tag, krn, m0 = synthetic.multigrain(n=10, L=15.0, grains=2, cone_deg=20.0, gb=2.0, seed=12)
    with _native.Mesh(X, T, tag, krn) as M:
        M.set_state(m0, None, m0)
        M.autotune(_native.solver_params(hdir=[0.0, 0.0, 1.0]))
        assert M.info()["pcg_variant"] in (1, 2)
