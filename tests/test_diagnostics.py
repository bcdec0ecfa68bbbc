"""The energy diagnostics (the reference's exani / external / hmag scripts) on the host:
their tables, analytic values and the field energy, with the library's mesh replaced by an
oracle-backed stand-in so that the whole script path runs without a GPU.  The values are
the reference's own known answers (tests/data/{exani,external,hmag} of the reference)."""

import numpy as np
import pytest

import oracle as O
from mammos_mumag import diagnostics, fly
from mammos_mumag.simulation import Simulation


class OracleMesh:
    """Stands in for ``_native.Mesh`` in these tests: the same calls, answered by the oracle."""

    def __init__(self, X, T, tag, krn, **kw):
        self.P = O.Problem(X, T, tag, krn)
        self.m = self.u = self.g = None

    def meas(self):
        return self.P.meas.copy(), self.P.V

    def set_state(self, m, u, mbar):
        self.m = np.asarray(m, np.float64).copy()
        self.u = np.zeros(self.P.N) if u is None else np.asarray(u, np.float64).copy()

    def energy_grad(self, h, sp):
        E, gp, self.u, self.g = O.total_eg(self.P, self.m, h, list(sp.hdir), self.u, sp.tol_u, hmag_on=sp.hmag_on)
        return E, gp, 0

    def get_state(self):
        return self.m.copy(), self.u.copy(), self.g.copy()

    def close(self):
        pass


@pytest.fixture
def sim(monkeypatch, tmp_path, cube_mesh, golden, energies):
    monkeypatch.setattr(diagnostics._native, "Mesh", OracleMesh)
    X, T, tag = cube_mesh
    fly.write_mesh(tmp_path / "cube.fly", X, T, tag)
    (tmp_path / "cube.krn").write_text(energies["krn"]["exani"])
    (tmp_path / "cube.p2").write_text(energies["p2"]["external"])
    return Simulation(mesh_filepath=tmp_path / "cube.fly", materials_filepath=tmp_path / "cube.krn",
                      parameters_filepath=tmp_path / "cube.p2")


def _check(out, gold, rel):
    assert set(out) == set(gold)
    for k, v in gold.items():
        assert out[k] == pytest.approx(v, rel=rel[k] if isinstance(rel, dict) else rel), k


def test_exani_tables(sim, tmp_path, energies):
    sim.run_exani(outdir=tmp_path / "exani")
    _check(diagnostics.read_csv(tmp_path / "exani" / "out_vortex.csv"), energies["exani_vortex"], 1e-11)
    _check(diagnostics.read_csv(tmp_path / "exani" / "out_uniform.csv"), energies["exani_uniform"], 1e-11)
    text = (tmp_path / "exani" / "out_uniform.csv").read_text()
    assert text.startswith("Magnetocrystalline anisotropy energy density of uniformly magnetized sample in direction "
                           "[0.0, 0.0, 1.0].\nname,value,explanation\nE_gradient,")
    assert not text.endswith("\n")
    assert (tmp_path / "exani" / "info.json").exists()


def test_external_table(sim, tmp_path, energies):
    sim.run_external(outdir=tmp_path / "external")
    _check(diagnostics.read_csv(tmp_path / "external" / "out.csv"), energies["external"], 1e-9)
    first = (tmp_path / "external" / "out.csv").read_text().splitlines()[0]
    assert first == "Zeeman energy density for an external field of mu_0 Hext 1.1 (T)."


def test_hmag_table_and_fields(sim, tmp_path, cube_mesh, energies):
    sim.run_hmag(outdir=tmp_path / "hmag")
    # E_field and E_gradient: the reference's potential came from escript's own solver;
    # E_analytic is Js^2 / 6 mu0
    _check(diagnostics.read_csv(tmp_path / "hmag" / "out.csv"), energies["hmag"],
           {"E_field": 1e-8, "E_gradient": 1e-9, "E_analytic": 1e-14})
    d = diagnostics.vtu.read_point_data(tmp_path / "hmag" / "out_hmag.vtu", ("m", "U", "h_nodes", "h"))
    X, T, tag = cube_mesh
    assert d["U"].size == len(X) and d["m"].size == 3 * len(X) and d["h_nodes"].size == 3 * len(X)
    h = d["h"].reshape(-1, 3)
    assert h.shape[0] == len(T)
    # the cube is magnetised along +z: inside it the demagnetising field points along -z,
    # about Js/3 for a cube (the mean over the magnet's cells)
    magnet = diagnostics.element_js(tag, O.read_krn_rows(energies["krn"]["hmag"])) > 0
    assert -0.8 * 1.61 / 3 > h[magnet, 2].mean() > -1.2 * 1.61 / 3


def test_field_energy_of_oracle_potential(cube_mesh, energies):
    """E_field (scripts/hmag.py:142) from the oracle's potential of the uniform state."""
    X, T, tag = cube_mesh
    krn = O.read_krn_rows(energies["krn"]["hmag"])
    P = O.Problem(X, T, tag, krn)
    m = O.initial_m_uniform(P, [0.0, 0.0, 1.0])
    u, _ = O.pcg(P.S, P.diagS, P.divergence(m), np.zeros(P.N), 1e-12)
    ef = diagnostics.field_energy(X, T, tag, krn, u, m, P.V) / diagnostics.MU0_OUT
    assert ef == pytest.approx(energies["hmag"]["E_field"], rel=1e-9)


def test_vortex_and_analytic_helpers(cube_mesh, energies):
    X, T, tag = cube_mesh
    krn = O.read_krn_rows(energies["krn"]["exani"])
    P = O.Problem(X, T, tag, krn)
    m, k = diagnostics.vortex_m(X, P.meas, P.V)
    mo, ko = O.vortex_m(P)
    assert k == ko and np.array_equal(m, mo)
    ea = diagnostics.anisotropy_energy(krn[0], [0.0, 0.0, 1.0]) / diagnostics.MU0_OUT
    assert ea == pytest.approx(energies["exani_uniform"]["E_analytic"], rel=1e-15)


def test_mapping_tables(sim, tmp_path, energies):
    """The mapping script's five tables.  The reference's values came from float32 JAX; its
    own test compares with np.allclose, which FP64 values meet; the FP64 rows also match
    the FP64 diagnostics (exani, external, hmag) of the same reference run."""
    sim.run_mapping(outdir=tmp_path / "mapping")
    for key, gold in energies["mapping"].items():
        out = diagnostics.read_csv(tmp_path / "mapping" / f"out_{key}.csv")
        assert set(out) == set(gold)
        for k, v in gold.items():
            assert np.allclose(out[k], v), (key, k)
    d = {k: diagnostics.read_csv(tmp_path / "mapping" / f"out_{k}.csv") for k in energies["mapping"]}
    assert d["anisotropy"]["E_jax"] == pytest.approx(energies["exani_uniform"]["E_gradient"], rel=1e-11)
    assert d["exchange"]["E_jax"] == pytest.approx(energies["exani_vortex"]["E_gradient"], rel=1e-11)
    assert d["zeeman"]["E_jax"] == pytest.approx(energies["external"]["E_gradient"], rel=1e-9)
    assert d["hmag"]["E_jax"] == pytest.approx(energies["hmag"]["E_gradient"], rel=1e-9)
    tot = d["zeeman"]["E_jax"] + d["anisotropy"]["E_jax"] + d["hmag"]["E_jax"]
    assert d["energy"]["E_jax"] == pytest.approx(tot, rel=1e-9)
    assert (tmp_path / "mapping" / "out_stats.txt").exists()


def test_runner_dispatches_scripts(monkeypatch, tmp_path, cube_mesh, energies):
    """``python -m mammos_mumag.runner <name> <script>``: the script table and its errors."""
    from mammos_mumag import runner

    monkeypatch.setattr(diagnostics._native, "Mesh", OracleMesh)
    X, T, tag = cube_mesh
    fly.write_mesh(tmp_path / "c.fly", X, T, tag)
    (tmp_path / "c.krn").write_text(energies["krn"]["exani"])
    out = runner.run_script("exani", tmp_path, "c")
    assert out["uniform"]["E_gradient"] == pytest.approx(energies["exani_uniform"]["E_gradient"], rel=1e-11)
    assert (tmp_path / "c_vortex.csv").exists()
    with pytest.raises(ValueError, match="not provided"):
        runner.run_script("store", tmp_path, "c")


def test_materials_and_magnetization_dumps(sim, tmp_path, cube_mesh, energies):
    """run_materials: per-element u, K (= K1), Js and A (= mu0 A) of the magnet, zero in the
    air and shell; run_magnetization: the .p2 initial state, masked to the magnet's nodes."""
    X, T, tag = cube_mesh
    krn = O.read_krn_rows(energies["krn"]["exani"])
    sim.run_materials(outdir=tmp_path / "mat")
    d = diagnostics.vtu.read_point_data(tmp_path / "mat" / "out_mat.vtu", ("u", "K", "Js", "A"))
    magnet = diagnostics.element_js(tag, krn) > 0
    assert magnet.any() and not magnet.all()
    assert np.allclose(d["Js"][magnet], krn[0][4]) and np.all(d["Js"][~magnet] == 0)
    assert np.allclose(d["K"][magnet], krn[0][2], rtol=1e-12)
    assert np.allclose(d["A"][magnet], diagnostics.MU0_SCRIPT * krn[0][5], rtol=1e-12)
    assert np.allclose(d["u"].reshape(-1, 3)[magnet], [0.0, 0.0, 1.0])
    sim.run_magnetization(outdir=tmp_path / "mag")
    m = diagnostics.vtu.read_point_data(tmp_path / "mag" / "out.0000.vtu", ("m",))["m"]
    P = O.Problem(X, T, tag, krn)
    np.testing.assert_allclose(m, O.initial_m_uniform(P, [0.0, 0.0, 1.0]), atol=1e-6)  # %e text
