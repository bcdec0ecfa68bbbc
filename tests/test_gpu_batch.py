"""Batched persistent launch: several meshes of uneven size stepped together in one
cooperative launch (CTA groups per mesh).  Each mesh must follow its standalone run."""

import numpy as np
import pytest

from mammos_mumag import _native, synthetic

pytestmark = pytest.mark.gpu


def _meshes():
    specs = [dict(n=5, L=15.0, grains=1, seed=1), dict(n=8, L=20.0, grains=3, seed=2), dict(n=11, L=26.0, grains=5, seed=3)]
    return [synthetic.multigrain(n=s["n"], L=s["L"], grains=s["grains"], cone_deg=30.0, gb=2.0, seed=s["seed"])
            for s in specs]


def test_batch_groups_and_single_step():
    data = _meshes()
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    ms = [_native.Mesh(X, T, tag, krn) for X, T, tag, krn, _ in data]
    try:
        for M, (_, _, _, _, m0) in zip(ms, data):
            M.set_state(m0, None, m0)
        alone = []
        for M, (_, _, _, _, m0) in zip(ms, data):
            alone.append(M.minimize(0.5, sp))
            M.set_state(m0, None, m0)
        with _native.Batch(ms) as B:
            g = B.groups()
            assert g[0] == 0 and (np.diff(g) >= 1).all()
            assert np.diff(g)[2] >= np.diff(g)[0]  # the largest mesh gets at least as many CTAs
            res = B.minimize(0.5, sp)
        for r, a in zip(res, alone):
            assert r["status"] == 0
            assert r["energy"] == pytest.approx(a["energy"], rel=1e-6)
            assert r["mh"] == pytest.approx(a["mh"], rel=1e-4)
    finally:
        for M in ms:
            M.close()


@pytest.mark.parametrize("mixed_mesh", [False, True])
def test_batch_loop_matches_standalone(mixed_mesh):
    data = _meshes()
    d = np.radians(1.0)
    sp = _native.solver_params(hdir=[np.sin(d), 0.0, np.cos(d)])
    precs = [0, 1 if mixed_mesh else 0, 0]
    sweep = (3.0, -3.0, -0.5, 0.4, -2.0)
    ms = [_native.Mesh(X, T, tag, krn, precision=p) for (X, T, tag, krn, _), p in zip(data, precs)]
    try:
        alone = []
        for M, (_, _, _, _, m0) in zip(ms, data):
            M.set_state(m0, None, m0)
            alone.append(M.loop(*sweep, sp)[0])
        for M, (_, _, _, _, m0) in zip(ms, data):
            M.set_state(m0, None, m0)
        with _native.Batch(ms) as B:
            out = B.loop(*sweep, sp)
        for (rows, steps), ref in zip(out, alone):
            assert rows.shape == ref.shape
            np.testing.assert_array_equal(rows[:, 1], ref[:, 1])
            np.testing.assert_allclose(rows[:, 2], ref[:, 2], rtol=2e-5)  # NCG stopping rule
            np.testing.assert_allclose(rows[:, 3], ref[:, 3], rtol=1e-8)
            assert all(s["status"] == 0 for s in steps)
    finally:
        for M in ms:
            M.close()
