"""The failure path of the persistent kernel, exercised without a GPU fault: every grid
barrier waits for one arrival that never comes (the mm_debug_stall_barriers test hook), so
each wait runs into its bound, the kernel records MM_TIMEOUT and returns, the call reports
it, and the mesh works normally afterwards."""

import time

import numpy as np
import pytest

from mammos_mumag import _native, synthetic

pytestmark = pytest.mark.gpu


def test_stalled_barrier_times_out_and_mesh_recovers():
    X, T, tag, krn, m0 = synthetic.multigrain(n=8, L=12.0, grains=2, cone_deg=20.0, gb=2.0, seed=21)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    with _native.Mesh(X, T, tag, krn) as M:
        M.set_state(m0, None, m0)
        E0, g0, _ = M.energy_grad(0.2, sp)
        M.debug_stall_barriers(1)
        M.set_state(m0, None, m0)
        t = time.perf_counter()
        with pytest.raises(_native.NativeError) as e:
            M.energy_grad(0.2, sp)
        waited = time.perf_counter() - t
        assert e.value.status == _native.MM_TIMEOUT
        assert waited < 60.0
        M.debug_stall_barriers(0)
        M.set_state(m0, None, m0)
        E1, g1, _ = M.energy_grad(0.2, sp)
    assert E1 == E0 and np.array_equal(g1, g0)
