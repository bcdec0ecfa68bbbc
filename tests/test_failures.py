"""Failure paths made on the host, as the reference's users meet them: corrupt input files,
non-finite inputs, bad options.  Each fails before any device work, so these run (and mean
the same) with or without a GPU; the reference surfaces such failures as
``RuntimeError("Simulation has failed. ...")`` from its subprocess wrapper
(``simulation.py:410-431``), and so does the in-process drop-in."""

import numpy as np
import pytest

from mammos_mumag import _native, fly, runner, synthetic
from mammos_mumag.materials import Materials
from mammos_mumag.parameters import Parameters
from mammos_mumag.simulation import Simulation

KRN = [[0.0, 0.0, 4.9e6, 0.0, 1.61, 8e-11]]


def _fly(tmp_path, text):
    p = tmp_path / "bad.fly"
    p.write_text(text)
    return p


def test_corrupt_fly_files_are_refused(tmp_path):
    good = "m\n3D-nodes 4\n1 1 0 0 0 0\n2 2 0 1 0 0\n3 3 0 0 1 0\n4 4 0 0 0 1\nTet4 1\n1 1 1 2 3 4\n"
    X, T, tag = fly.read_mesh(_fly(tmp_path, good))
    assert X.shape == (4, 3) and T.tolist() == [[0, 1, 2, 3]] and tag.tolist() == [1]
    with pytest.raises(ValueError, match="nodes"):
        fly.read_mesh(_fly(tmp_path, "m\nnodes\n"))
    with pytest.raises(ValueError, match="Tet4"):
        fly.read_mesh(_fly(tmp_path, good.replace("Tet4 1", "Hex8 1")))
    with pytest.raises(ValueError, match="undefined node"):
        fly.read_mesh(_fly(tmp_path, good.replace("1 1 1 2 3 4", "1 1 1 2 3 9")))


def test_loop_failure_surfaces_as_simulation_error(tmp_path):
    bad = _fly(tmp_path, "m\n3D-nodes 1\n1 1 0 0 0 0\nTet4 1\n1 1 1 2 3 4\n")
    (tmp_path / "m.krn").write_text("0 0 4.9e6 0 1.61 8e-11 1.0 0.0\n")
    sim = Simulation(mesh_filepath=bad, materials_filepath=tmp_path / "m.krn", parameters=Parameters())
    with pytest.raises(RuntimeError, match="Simulation has failed. Exit with error"):
        sim.run_loop(outdir=tmp_path / "out")
    with pytest.raises(AttributeError, match="parameters"):
        Simulation(mesh_filepath=bad, materials=Materials(domains=[{"Ms": 1e6}])).run_loop(outdir=tmp_path / "o2")


@pytest.mark.parametrize("what", ["nan", "inf"])
def test_non_finite_coordinates_are_refused(what):
    X, T = synthetic.cube_grid(2, 4.0)
    X = X.copy()
    X[3, 1] = float(what)
    with pytest.raises(_native.NativeError) as ei:
        _native.Mesh(X, T, np.ones(len(T), np.int32), KRN)
    assert ei.value.status == _native.MM_BAD_INPUT and "non-finite" in str(ei.value)


def test_malformed_p2_is_refused(tmp_path):
    p = tmp_path / "x.p2"
    p.write_text("[initial state]\nmx = 0\nmy = 0\nmz = 1\n[field]\nhstart = one\n")
    with pytest.raises((KeyError, ValueError)):
        runner.read_script_params(p)
