"""The reference-facing API end to end on the GPU: Simulation.run_loop writes the files
the reference's loop script writes, with the golden's numbers."""

import json

import numpy as np
import pytest

from mammos_mumag import hysteresis, mesh, vtu
from mammos_mumag.simulation import Simulation

pytestmark = pytest.mark.gpu


def test_simulation_run_loop_reproduces_golden(golden, tmp_path):
    sim = Simulation(
        mesh_filepath=mesh.CUBE_20_nm,
        materials_filepath=golden / "loop_cube.krn",
        parameters_filepath=golden / "loop_cube.p2",
    )
    sim.run_loop(outdir=tmp_path, name="cube")
    gold = np.loadtxt(golden / "loop_cube.dat")
    out = np.loadtxt(tmp_path / "cube.dat")
    assert np.allclose(gold, out)  # the reference's own check (tests/test_loop.py:21-23)
    np.testing.assert_allclose(out, gold, rtol=1e-9)
    vtus = sorted(p.name for p in tmp_path.glob("*.vtu"))
    assert vtus == ["cube_0001.vtu"]
    m = vtu.read_point_data(tmp_path / "cube_0001.vtu")["m"].reshape(-1, 3)
    assert np.allclose(np.load(golden / "loop_cube_0001.npz")["m"], m)
    for f in ("cube.fly", "cube.krn", "cube.p2", "cube_stats.txt", "info.json"):
        assert (tmp_path / f).exists(), f
    assert "mammos_mumag_version" in json.loads((tmp_path / "info.json").read_text())


def test_hysteresis_run(tmp_path):
    mu0 = 4e-7 * np.pi
    res = hysteresis.run(Ms=1.28e6, A=7.7e-12, K1=4.3e6, mesh_filepath=mesh.CUBE_20_nm,
                         hstart=2.0 / mu0, hfinal=-2.0 / mu0, hnsteps=4, outdir=tmp_path / "h")
    assert len(res.H) == 5
    assert res.H[0] == pytest.approx(2.0 / mu0, rel=1e-6)
    assert (res.M > 0).all()  # a 7.6 T anisotropy field: no switching at -2 T
    assert list(res.configurations) == [1]
    assert res.dataframe.shape == (5, 4)


def test_failure_raises_runtime_error(tmp_path, golden):
    sim = Simulation(mesh_filepath=mesh.CUBE_20_nm, materials_filepath=golden / "io" / "cube.krn",
                     parameters_filepath=golden / "loop_cube.p2")
    sim.materials.domains = sim.materials.domains[:1]  # 1 row for 3 element tags
    with pytest.raises(RuntimeError, match="Simulation has failed"):
        sim.run_loop(outdir=tmp_path, name="bad")
