"""Device-resident state at the C ABI (mm_set_state_device / mm_get_state_device): the same
state as the host form, from and into device memory the caller owns.  The reference's
total_eg takes JAX device arrays (scripts/energies.py:67-99); a caller whose magnetisation
already lives on the GPU should not need a host round trip."""

import numpy as np
import pytest

from mammos_mumag import _native, synthetic

pytestmark = pytest.mark.gpu


def test_device_state_matches_host_state():
    import torch

    X, T, tag, krn, m0 = synthetic.multigrain(n=10, L=25.0, grains=3, cone_deg=20.0, gb=2.0, seed=4)
    rng = np.random.default_rng(3)
    u0 = rng.standard_normal(X.shape[0]) * 1e-3
    mb = np.roll(m0, 3)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    dev = torch.device("cuda:0")
    with _native.Mesh(X, T, tag, krn) as M:
        M.set_state(m0, u0, mb)
        Eh, gh, ith = M.energy_grad(0.3, sp)
        mh, uh, gfh = M.get_state()
        dm, du, dmb = (torch.from_numpy(a).to(dev) for a in (m0, u0, mb))
        torch.cuda.synchronize()
        M.set_state_device(dm.data_ptr(), du.data_ptr(), dmb.data_ptr())
        Ed, gd, itd = M.energy_grad(0.3, sp)
        om, ou, og = (torch.zeros(n, dtype=torch.float64, device=dev) for n in (3 * M.N, M.N, 3 * M.N))
        M.get_state_device(om.data_ptr(), ou.data_ptr(), og.data_ptr())
        assert Ed == Eh and ith == itd
        np.testing.assert_array_equal(gd, gh)
        np.testing.assert_array_equal(om.cpu().numpy(), mh)
        np.testing.assert_array_equal(ou.cpu().numpy(), uh)
        np.testing.assert_array_equal(og.cpu().numpy(), gfh)
        # u and mbar are optional, as in the host form (u = 0, mbar = m)
        M.set_state(m0, None, None)
        E0 = M.energy_grad(0.3, sp)[0]
        M.set_state_device(dm.data_ptr())
        assert M.energy_grad(0.3, sp)[0] == E0
        # a non-finite value is refused
        bad = dm.clone()
        bad[7] = float("nan")
        with pytest.raises(_native.NativeError, match="non-finite"):
            M.set_state_device(bad.data_ptr())
