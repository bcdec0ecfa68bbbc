"""The reference's energy known-answer scripts (exani, external, hmag, mapping) through
``Simulation.run_*`` on the GPU path, compared with the tables the reference itself wrote
(tests/data/{exani,external,hmag}/*.csv of the reference; the reference's tests compare them
with np.allclose, the bounds here are tighter)."""

import numpy as np
import pytest

from mammos_mumag import diagnostics, fly
from mammos_mumag.simulation import Simulation

pytestmark = pytest.mark.gpu


@pytest.fixture
def sim(tmp_path, cube_mesh, energies):
    X, T, tag = cube_mesh
    fly.write_mesh(tmp_path / "cube.fly", X, T, tag)
    (tmp_path / "cube.krn").write_text(energies["krn"]["exani"])
    (tmp_path / "cube.p2").write_text(energies["p2"]["external"])
    return Simulation(mesh_filepath=tmp_path / "cube.fly", materials_filepath=tmp_path / "cube.krn",
                      parameters_filepath=tmp_path / "cube.p2")


def _check(out, gold, rel):
    assert set(out) == set(gold)
    for k, v in gold.items():
        assert np.allclose(out[k], v)  # the reference's own test bound
        assert out[k] == pytest.approx(v, rel=rel[k] if isinstance(rel, dict) else rel), k


def test_exani_on_gpu(sim, tmp_path, energies):
    sim.run_exani(outdir=tmp_path / "exani")
    _check(diagnostics.read_csv(tmp_path / "exani" / "out_vortex.csv"), energies["exani_vortex"], 1e-11)
    _check(diagnostics.read_csv(tmp_path / "exani" / "out_uniform.csv"), energies["exani_uniform"], 1e-11)


def test_external_on_gpu(sim, tmp_path, energies):
    sim.run_external(outdir=tmp_path / "external")
    _check(diagnostics.read_csv(tmp_path / "external" / "out.csv"), energies["external"], 1e-9)


def test_hmag_on_gpu(sim, tmp_path, cube_mesh, energies):
    sim.run_hmag(outdir=tmp_path / "hmag")
    _check(diagnostics.read_csv(tmp_path / "hmag" / "out.csv"), energies["hmag"],
           {"E_field": 1e-8, "E_gradient": 1e-9, "E_analytic": 1e-14})
    X, T, tag = cube_mesh
    d = diagnostics.vtu.read_point_data(tmp_path / "hmag" / "out_hmag.vtu", ("U", "h_nodes", "h"))
    assert d["U"].size == len(X) and d["h_nodes"].size == 3 * len(X) and d["h"].size == 3 * len(T)


def test_mapping_on_gpu(sim, tmp_path, energies):
    """The mapping tables (the reference's are float32 JAX: np.allclose, its own bound; the
    FP64 rows also against the FP64 known answers of the other scripts)."""
    sim.run_mapping(outdir=tmp_path / "mapping")
    d = {k: diagnostics.read_csv(tmp_path / "mapping" / f"out_{k}.csv") for k in energies["mapping"]}
    for key, gold in energies["mapping"].items():
        for k, v in gold.items():
            assert np.allclose(d[key][k], v), (key, k)
    assert d["anisotropy"]["E_jax"] == pytest.approx(energies["exani_uniform"]["E_gradient"], rel=1e-11)
    assert d["exchange"]["E_jax"] == pytest.approx(energies["exani_vortex"]["E_gradient"], rel=1e-11)
    assert d["zeeman"]["E_jax"] == pytest.approx(energies["external"]["E_gradient"], rel=1e-9)
    assert d["hmag"]["E_jax"] == pytest.approx(energies["hmag"]["E_gradient"], rel=1e-9)
