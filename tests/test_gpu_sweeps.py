"""Whole field sweeps through the coercive field, GPU against the FP64 oracle.

The reference records no loop that crosses the coercive field, and its bare-box boundary
branch (every synthetic workload's) has no golden, so the pins here are the FP64 oracle's own
sweeps (``tests/golden/sweep_*.npz``, made by ``tests/golden/make_sweeps.py``; the oracle is
pinned to the reference's goldens by ``tests/test_oracle_golden.py``):

* the single grain (20 nm, 16^3 x 6 tets, +8 -> -8 T in 0.2 T steps, all 81 steps) and the
  multigrain cube (80 nm, 32^3 x 6 tets, 8 grains + boundary phase, 161 steps);
* FP64 on the GPU: the same rows (field values bit for bit, mh and energy to the NCG
  stopping rule's tolerance) and Hc, Mr within 1e-3 relative;
* mixed precision, the two-level preconditioner and the learned warm start: Hc and Mr
  within 1 % of the oracle's (the contract's bar for the mixed-precision path).
"""

import json
import pathlib
import sys

import numpy as np
import pytest

from mammos_mumag import _native, learned
from mammos_mumag.hysteresis import coercivity_remanence

ROOT = pathlib.Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "tests" / "golden"))
import make_sweeps  # noqa: E402

pytestmark = pytest.mark.gpu


def _fixture(name):
    f = np.load(ROOT / "tests" / "golden" / f"sweep_{name}.npz")
    assert json.loads(str(f["params"])) == make_sweeps.CASES[name]
    return f["rows"], f["stats"], float(f["hc"]), float(f["mr"])


def _run(name, precision=_native.PREC_FP64, coarse=0, model=None):
    X, T, tag, krn, m0, par = make_sweeps.build_case(name)
    with _native.Mesh(X, T, tag, krn, precision=precision, coarse_box_nodes=coarse) as M:
        if model is not None:
            M.set_warm_start(_native.WARM_LEARNED, model)
        M.set_state(m0, None, m0)
        rows, steps = M.loop(par["hstart"], par["hfinal"], par["hstep"], par["mstep"], par["mfinal"],
                             _native.solver_params(hdir=par["hdir"]))
    return rows, steps


@pytest.mark.parametrize("name", ["single", "multigrain"])
def test_fp64_sweep_matches_oracle(name):
    rows_o, _, hc_o, mr_o = _fixture(name)
    rows, steps = _run(name)
    assert all(s["status"] == 0 for s in steps)
    assert rows.shape == rows_o.shape
    np.testing.assert_array_equal(rows[:, 1], rows_o[:, 1])  # cumulative field values
    np.testing.assert_array_equal(rows[:, 0], rows_o[:, 0])  # snapshot counter
    # loop tolerance of the NCG stopping rule (tests/test_gpu_parity.py), through switching
    np.testing.assert_allclose(rows[:, 2], rows_o[:, 2], rtol=2e-5, atol=2e-5)
    np.testing.assert_allclose(rows[:, 3], rows_o[:, 3], rtol=1e-7)
    hc, mr = coercivity_remanence(rows)
    assert np.isfinite(hc_o) and np.isfinite(mr_o), "the oracle's sweep must switch"
    assert abs(hc - hc_o) <= 1e-3 * hc_o
    assert abs(mr - mr_o) <= 1e-3 * abs(mr_o)


@pytest.fixture(scope="module")
def model():
    """A network trained quickly on plain loops of two 16^3 multigrain cubes (the learned
    start's family); its quality does not matter here, only that the sweeps it starts reach
    the same loop."""
    spec = learned.LoopSpec(max_steps=20)
    feats, targets = learned.collect([900, 901], spec, samples=8000)
    net, _ = learned.train(feats, targets, epochs=4)
    yield net
    net.close()


@pytest.mark.parametrize("name", ["single", "multigrain"])
@pytest.mark.parametrize("variant", ["mixed", "coarse", "mixed_coarse", "learned_mixed", "learned_mixed_coarse"])
def test_fast_paths_hc_mr_within_one_percent_of_oracle(name, variant, model):
    _, _, hc_o, mr_o = _fixture(name)
    prec = _native.PREC_MIXED if "mixed" in variant else _native.PREC_FP64
    coarse = (64 if name == "single" else 256) if "coarse" in variant else 0
    rows, steps = _run(name, prec, coarse, model if "learned" in variant else None)
    assert all(s["status"] == 0 for s in steps)
    hc, mr = coercivity_remanence(rows)
    assert abs(hc - hc_o) <= 0.01 * hc_o, (hc, hc_o)
    assert abs(mr - mr_o) <= 0.01 * abs(mr_o), (mr, mr_o)
