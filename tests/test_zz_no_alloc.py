"""The allocation-free Poisson solve (mm_poisson_pcg_noalloc) through the C ABI.

Callers that cannot allocate device memory (plug-ins whose host application owns every
device byte, services that forbid allocation while serving) solve the magnetostatic Poisson system through
this entry point with their own device buffers; its scratch is a static device array.  The
solution must match the one the mesh path computes inside an energy evaluation, on two calls
in a row (the second call reuses the static array the first one left behind).  This file
sorts last so that a run that stops at the first failure has run every other test first.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from mammos_mumag import _native

pytestmark = pytest.mark.gpu


def _csr_of(M, which):
    r, c, v = M.operator(which)
    return sp.csr_matrix((v, (r, c)), shape=(M.N, M.N))


def test_noalloc_pcg_matches_mesh_path_twice(cube_mesh, golden):
    import torch

    X, T, tag = cube_mesh
    krn = O.read_krn_rows((golden / "loop_cube.krn").read_text())
    rng = np.random.default_rng(4)
    with _native.Mesh(X, T, tag, krn) as M:
        S = _csr_of(M, 0)
        S.sort_indices()
        Dk = [_csr_of(M, 8 + k) for k in range(3)]
        meas, _ = M.meas()
        mask = meas > 0
        dev = torch.device("cuda:0")
        rp = torch.from_numpy(S.indptr.astype(np.int32)).to(dev)
        ci = torch.from_numpy(S.indices.astype(np.int32)).to(dev)
        av = torch.from_numpy(S.data.astype(np.float64)).to(dev)
        sp_ = _native.solver_params(hdir=[0.0, 0.0, 1.0])
        for call in range(2):
            m = rng.standard_normal((M.N, 3)) + np.array([0.0, 0.0, 1.5 + call])
            m = O.normalize_vectors((m * mask[:, None]).ravel())
            # the existing entry point: one energy evaluation solves S u = b from u = 0
            M.set_state(m, None, m)
            M.energy_grad(0.0, sp_)
            _, u_ref, _ = M.get_state()
            b = Dk[0] @ m[0::3] + Dk[1] @ m[1::3] + Dk[2] @ m[2::3]
            bd = torch.from_numpy(b).to(dev)
            xd = torch.zeros(M.N, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            it = _native.poisson_pcg_noalloc(M.N, S.nnz, rp.data_ptr(), ci.data_ptr(), av.data_ptr(), bd.data_ptr(),
                                             xd.data_ptr(), tol=1e-10, max_iter=10000,
                                             stream=torch.cuda.current_stream().cuda_stream)
            x = xd.cpu().numpy()
            assert it > 10
            # both solves meet |r| <= 1e-10 |b|; their solutions agree far inside the 1e-6
            # relative bar the energy/field parity tests use
            assert np.abs(x - u_ref).max() <= 1e-6 * np.abs(u_ref).max(), call
            assert np.abs(S @ x - b).max() <= 1e-8 * np.abs(b).max()


def test_noalloc_rejects_oversize_and_bad_structure():
    import torch

    dev = torch.device("cuda:0")
    one = torch.zeros(2, dtype=torch.int32, device=dev)
    v = torch.ones(1, dtype=torch.float64, device=dev)
    with pytest.raises(_native.NativeError, match="65536"):
        _native.poisson_pcg_noalloc(70000, 1, one.data_ptr(), one.data_ptr(), v.data_ptr(), v.data_ptr(),
                                    v.data_ptr())
    # one row whose only column points outside the matrix: reported, not dereferenced
    rp = torch.tensor([0, 1], dtype=torch.int32, device=dev)
    ci = torch.tensor([5], dtype=torch.int32, device=dev)
    x = torch.zeros(1, dtype=torch.float64, device=dev)
    with pytest.raises(_native.NativeError, match="out of range"):
        _native.poisson_pcg_noalloc(1, 1, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), v.data_ptr(), x.data_ptr())
    # rows whose diagonal is missing, zero or not finite: the Jacobi preconditioner would
    # divide by it, so the call refuses them before iterating and reports 0 iterations
    rp2 = torch.tensor([0, 1, 2], dtype=torch.int32, device=dev)
    b2 = torch.ones(2, dtype=torch.float64, device=dev)
    x2 = torch.zeros(2, dtype=torch.float64, device=dev)
    cases = {
        "missing": ([1, 0], [2.0, 2.0]),   # row 0 holds only column 1
        "zero": ([0, 1], [0.0, 2.0]),
        "nan": ([0, 1], [float("nan"), 2.0]),
        "inf": ([0, 1], [2.0, float("inf")]),
    }
    for name, (cols, vals) in cases.items():
        ci2 = torch.tensor(cols, dtype=torch.int32, device=dev)
        av2 = torch.tensor(vals, dtype=torch.float64, device=dev)
        st, it = _native.poisson_pcg_noalloc(2, 2, rp2.data_ptr(), ci2.data_ptr(), av2.data_ptr(), b2.data_ptr(),
                                             x2.data_ptr(), raise_error=False)
        assert st == _native.MM_BAD_INPUT, name
        assert it == 0, name
        assert "diagonal" in _native.load().mm_last_error().decode(), name
        assert torch.all(x2 == 0), name


def _laplacian_1d(n):
    """The 1-D Dirichlet Laplacian (tridiagonal 2, -1): CG needs about n/2 iterations."""
    main = 2.0 * np.ones(n)
    off = -np.ones(n - 1)
    A = sp.diags([off, main, off], [-1, 0, 1], format="csr")
    A.sort_indices()
    return A


def test_noalloc_max_iter_caps_an_unconverged_solve():
    """max_iter stops the solve early, as the reference's cg does: the call succeeds, reports
    exactly max_iter iterations and returns the CG iterate after them (the oracle's CG with
    the same cap), whose residual is still far above the tolerance."""
    import torch

    n, cap = 3000, 7
    A = _laplacian_1d(n)
    rng = np.random.default_rng(11)
    b = rng.standard_normal(n)
    dev = torch.device("cuda:0")
    rp = torch.from_numpy(A.indptr.astype(np.int32)).to(dev)
    ci = torch.from_numpy(A.indices.astype(np.int32)).to(dev)
    av = torch.from_numpy(A.data.astype(np.float64)).to(dev)
    bd = torch.from_numpy(b).to(dev)
    xd = torch.zeros(n, dtype=torch.float64, device=dev)
    it = _native.poisson_pcg_noalloc(n, A.nnz, rp.data_ptr(), ci.data_ptr(), av.data_ptr(), bd.data_ptr(),
                                     xd.data_ptr(), tol=1e-10, max_iter=cap)
    assert it == cap
    x = xd.cpu().numpy()
    xo, ko = O.pcg(A, A.diagonal(), b, np.zeros(n), 1e-10, maxiter=cap)
    assert ko == cap
    # the same iterate in another arrangement of the same recurrences: rounding-level agreement
    assert np.abs(x - xo).max() <= 1e-10 * np.abs(xo).max()
    assert np.linalg.norm(A @ x - b) > 1e-3 * np.linalg.norm(b)


def test_noalloc_barrier_timeout_then_recovers():
    """Every wait of the kernel is bounded: with the test hook making each grid barrier wait
    for an arrival that never comes, the call gives up after about two seconds and returns
    MM_TIMEOUT (no fault, no hang); with the hook cleared the next call solves normally."""
    import torch

    n = 2000
    A = _laplacian_1d(n)
    b = np.random.default_rng(12).standard_normal(n)
    dev = torch.device("cuda:0")
    rp = torch.from_numpy(A.indptr.astype(np.int32)).to(dev)
    ci = torch.from_numpy(A.indices.astype(np.int32)).to(dev)
    av = torch.from_numpy(A.data.astype(np.float64)).to(dev)
    bd = torch.from_numpy(b).to(dev)
    xd = torch.zeros(n, dtype=torch.float64, device=dev)
    args = (n, A.nnz, rp.data_ptr(), ci.data_ptr(), av.data_ptr(), bd.data_ptr(), xd.data_ptr())
    _native.noalloc_stall_barriers(1)
    try:
        st, it = _native.poisson_pcg_noalloc(*args, raise_error=False)
    finally:
        _native.noalloc_stall_barriers(0)
    assert st == _native.MM_TIMEOUT
    assert it == 0  # the first barrier never opened: nothing was iterated
    xd.zero_()
    it = _native.poisson_pcg_noalloc(*args, tol=1e-10, max_iter=10000)
    assert 0 < it < 10000
    x = xd.cpu().numpy()
    # the stop test reads the recursively updated residual; the true one agrees to rounding
    # (condition number ~1e6 here)
    assert np.linalg.norm(A @ x - b) <= 1e-8 * np.linalg.norm(b)
