"""The C ABI library loads, exports what include/mumag_b200.h declares, and its host-only
mesh utilities (RCM order, element colouring) are correct.  No GPU needed."""

import re

import numpy as np
import pytest

from mammos_mumag import _native, synthetic
from conftest import ROOT


def test_exports_match_header():
    lib = _native.load()
    header = (ROOT / "include" / "mumag_b200.h").read_text()
    declared = set(re.findall(r"\b(mm_[a-z_]+)\s*\(", header)) - {"mm_snapshot_cb"}
    assert declared == set(_native.EXPORTED)
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.mm_version().startswith(b"mumag_b200")


def test_rcm_is_a_permutation_and_reduces_bandwidth(cube_mesh):
    X, T, _ = cube_mesh
    N = X.shape[0]
    perm = _native.rcm_permutation(T, N)
    assert np.array_equal(np.sort(perm), np.arange(N))
    iperm = np.empty(N, np.int64)
    iperm[perm] = np.arange(N)
    pairs = np.stack(np.broadcast_arrays(T[:, :, None], T[:, None, :]), -1).reshape(-1, 2)
    bw0 = np.abs(pairs[:, 0] - pairs[:, 1]).max()
    bw1 = np.abs(iperm[pairs[:, 0]] - iperm[pairs[:, 1]]).max()
    assert bw1 < bw0 / 5


@pytest.mark.parametrize("n", [3, 6])
def test_colouring_is_conflict_free(n):
    X, T = synthetic.cube_grid(n, 10.0)
    col, nc = _native.color_elements(T, X.shape[0])
    assert col.min() == 0 and col.max() == nc - 1
    for c in range(nc):
        nodes = T[col == c].ravel()
        assert len(np.unique(nodes)) == len(nodes)
    # every node of a Freudenthal grid interior touches 24 tets: at least that many colours
    if n >= 3:
        assert nc >= 24


def test_bad_input_is_rejected():
    T = np.array([[0, 1, 2, 7]], np.int32)  # node 7 does not exist
    with pytest.raises(_native.NativeError) as ei:
        _native.rcm_permutation(T, 4)
    assert ei.value.status == _native.MM_BAD_INPUT
    assert "outside" in str(ei.value)


def test_no_device_is_reported_without_gpu():
    if _native.device_count() > 0:
        pytest.skip("a GPU is present")
    X, T = synthetic.cube_grid(2, 4.0)
    with pytest.raises(_native.NativeError) as ei:
        _native.Mesh(X, T, np.ones(len(T), np.int32), [[0, 0, 1e6, 0, 1.0, 1e-11]])
    assert ei.value.status == _native.MM_NO_DEVICE


@pytest.mark.parametrize("opt", [dict(stage_operators=2), dict(ctas_per_sm=4), dict(pcg_variant=3)])
def test_bad_options_are_rejected(opt):
    """Option values outside their range are refused before any device work (so also here)."""
    X, T = synthetic.cube_grid(2, 4.0)
    with pytest.raises(_native.NativeError) as ei:
        _native.Mesh(X, T, np.ones(len(T), np.int32), [[0, 0, 1e6, 0, 1.0, 1e-11]], **opt)
    assert ei.value.status == _native.MM_BAD_INPUT
    assert next(iter(opt)) in str(ei.value)


def test_host_preprocessing_independent_of_threads(monkeypatch):
    """The RCM order and the element colouring of a mesh large enough for several host
    threads are the same with one thread (MUMAG_HOST_THREADS=1) and with the default."""
    X, T = synthetic.cube_grid(52, 52.0)  # 148,877 nodes: the node passes use 2 threads or more
    perm, col = _native.rcm_permutation(T, X.shape[0]), _native.color_elements(T, X.shape[0])[0]
    monkeypatch.setenv("MUMAG_HOST_THREADS", "1")
    assert np.array_equal(perm, _native.rcm_permutation(T, X.shape[0]))
    assert np.array_equal(col, _native.color_elements(T, X.shape[0])[0])
