"""The preprocessing cache of mm_mesh_create (the counterpart of the reference's
scripts/store.py, which pickles escript's assembled arrays so that a rerun skips the set-up):
creating a mesh whose exact input was prepared before reuses the node order, SELL pattern,
colouring, boundary branch, aggregate boxes and coarse inverse.  A hit must give the same
operators and the same field step as the first creation; a changed input must not hit."""

import time

import numpy as np
import pytest

from mammos_mumag import _native, synthetic

pytestmark = pytest.mark.gpu


def test_cached_mesh_is_identical():
    X, T, tag, krn, m0 = synthetic.multigrain(n=24, L=60.0, grains=5, cone_deg=20.0, gb=2.0, seed=11)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    out = []
    for _ in range(2):
        t0 = time.perf_counter()
        with _native.Mesh(X, T, tag, krn, coarse_box_nodes=128) as M:
            dt = time.perf_counter() - t0
            ops = [M.operator(w) for w in (0, 1, 8)]
            box, nb = M.coarse()
            M.set_state(m0, None, m0)
            r = M.minimize(0.5, sp)
        out.append((dt, ops, box, nb, r))
    (d0, o0, b0, n0, r0), (d1, o1, b1, n1, r1) = out
    for a, b in zip(o0, o1):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(b0, b1)
    assert n0 == n1 and n0 > 0
    assert r0["energy"] == r1["energy"] and r0["pcg_iters"] == r1["pcg_iters"]
    # a different input: a node moved by a hundredth of a cell is prepared anew
    X2 = X.copy()
    X2[len(X2) // 2, 0] += 0.025
    with _native.Mesh(X2, T, tag, krn, coarse_box_nodes=128) as M:
        M.set_state(m0, None, m0)
        r2 = M.minimize(0.5, sp)
    assert r2["energy"] != r0["energy"]
