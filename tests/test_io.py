"""Host-side drop-in pieces: material/parameter files, .fly/.vtu I/O, synthetic meshes."""

import numpy as np
import pytest
from pydantic import ValidationError

import oracle as O
from mammos_mumag import fly, runner, synthetic, vtu
from mammos_mumag.materials import MaterialDomain, Materials
from mammos_mumag.parameters import Parameters
from conftest import ROOT


def test_materials_roundtrip(golden, tmp_path):
    mat = Materials(filepath=golden / "io" / "cube.krn")
    assert len(mat.domains) == 3
    assert mat.domains[0].K1 == 4.9e6 and mat.domains[0].Js == pytest.approx(1.61)
    mat.write_krn(tmp_path / "m.krn")
    mat.write_yaml(tmp_path / "m.yaml")
    for f in ("m.krn", "m.yaml"):
        back = Materials(filepath=tmp_path / f)
        for a, b in zip(mat.domains, back.domains):
            for k in ("theta", "phi", "K1", "K2", "Ms", "A"):
                assert getattr(a, k) == pytest.approx(getattr(b, k), rel=1e-12)
    yml = Materials(filepath=golden / "io" / "materials.yaml")
    assert yml.domains[0].Js == pytest.approx(1.61)
    # the .krn the loop reads carries the same numbers
    rows = runner.read_krn_rows(tmp_path / "m.krn")
    assert rows[0][:6] == pytest.approx([0.0, 0.0, 4.9e6, 0.0, 1.61, 8e-11])
    with pytest.raises(NotImplementedError):
        Materials().read(golden / "io" / "cube.p2")


def test_material_domain_types_and_validation():
    """As the reference's tests/test_materials_file.py:119-185: equal values give equal
    domains whatever their numeric type; the default domain is all zeros; values that are not
    numbers raise pydantic's ValidationError."""
    a = MaterialDomain(theta=0, phi=0, K1=1, K2=2, Ms=3, A=4)
    b = MaterialDomain(theta=0.0, phi=0.0, K1=np.float64(1), K2=2.0, Ms=np.int64(3), A=4.0)
    assert a == b
    assert MaterialDomain() == MaterialDomain(theta=0, phi=0, K1=0, K2=0, Ms=0, A=0)
    for bad in (dict(K1="K1"), dict(theta="x"), dict(A=[1, 2]), dict(Ms=None)):
        with pytest.raises(ValidationError):
            MaterialDomain(**bad)


def test_parameters_roundtrip_and_validation(golden, tmp_path):
    for bad in (1, 1.0, [1], [1, 2], [1, 2, 3, 4]):
        with pytest.raises(ValidationError):
            Parameters(m_vect=bad)
        with pytest.raises(ValidationError):
            Parameters(h_vect=bad)
    par = Parameters(m_vect=np.array([1, 2, 3]))
    assert par.m == [1.0 / np.sqrt(14), 2.0 / np.sqrt(14), 3.0 / np.sqrt(14)]
    par = Parameters(m=[1, 0, 0], hstart=8.0, hfinal=-1.5, hstep=-0.01, iter_max=5000)
    par.write_p2(tmp_path / "p.p2")
    par.write_yaml(tmp_path / "p.yaml")
    for f in ("p.p2", "p.yaml"):
        back = Parameters(filepath=tmp_path / f)
        for k in ("hstart", "hfinal", "hstep", "iter_max", "tol_fun", "precond_iter"):
            assert getattr(back, k) == getattr(par, k)
        assert back.m == pytest.approx(par.m)
    ref = Parameters(filepath=golden / "io" / "cube.p2")
    assert ref.h == pytest.approx(np.array([0.01745, 0, 0.99984]) / np.linalg.norm([0.01745, 0, 0.99984]))
    # the loop-script reader agrees with the oracle's restatement of scripts/tools.py
    p = runner.read_script_params(golden / "loop_cube.p2")
    q = O.read_params((golden / "loop_cube.p2").read_text())
    for k in ("hdir", "hstart", "hfinal", "hstep", "mstep", "mfinal", "tol_fun", "tol_u", "precond_iter", "hmag_on"):
        assert p[k] == q[k]


def test_fly_roundtrip(cube_mesh, tmp_path):
    X, T, tag = cube_mesh
    fly.write_mesh(tmp_path / "c.fly", X, T, tag)
    X2, T2, tag2 = fly.read_mesh(tmp_path / "c.fly")
    assert np.array_equal(X, X2) and np.array_equal(T, T2) and np.array_equal(tag, tag2)


def test_vtu_roundtrip(tmp_path):
    X, T = synthetic.cube_grid(2, 4.0)
    m = np.random.default_rng(1).standard_normal(3 * len(X))
    u = np.arange(len(X), dtype=float)
    vtu.write_vtu(tmp_path / "s_0001.vtu", X, T, np.ones(len(T)), {"m": m, "u": u})
    pd = vtu.read_point_data(tmp_path / "s_0001.vtu")
    np.testing.assert_allclose(pd["m"], m, rtol=1e-6)
    np.testing.assert_allclose(pd["u"], u, rtol=1e-6)


@pytest.mark.parametrize("n", [4, 7])
def test_synthetic_cube_takes_airbox_branch(n):
    X, T = synthetic.cube_grid(n, 20.0)
    assert X.shape[0] == (n + 1) ** 3 and T.shape[0] == 6 * n**3
    r = np.linalg.norm(X, axis=1)
    assert (r == r.max()).sum() == 8
    P = X[T]
    det = np.einsum("ij,ij->i", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))
    assert (det > 0).all()
    assert np.isclose(det.sum() / 6, 20.0**3)
    P_ = O.Problem(X, T, np.ones(len(T), np.int32), [[0, 0, 4.3e6, 0, 1.61, 7.7e-12]])
    assert P_.airbox and P_.bnd.sum() == (n + 1) ** 3 - (n - 1) ** 3


def test_multigrain_labels():
    X, T, tag, rows, m0 = synthetic.multigrain(n=12, L=40.0, grains=5, seed=3)
    assert len(rows) == len(np.unique(tag))
    assert tag.max() == 6 and (tag == 6).any()  # boundary phase present
    assert np.allclose(np.linalg.norm(m0.reshape(-1, 3), axis=1), 1.0)


def test_coercivity_remanence_definitions():
    """Hc = |mu0 H| at the first zero crossing of mh, Mr = mh at H = 0, linear interpolation;
    NaN when the loop does not reach them."""
    from mammos_mumag.hysteresis import coercivity_remanence

    h = np.array([1.0, 0.5, 0.0, -0.5, -1.0, -1.5])
    mh = np.array([1.0, 0.9, 0.8, 0.4, -0.6, -0.9])
    rows = np.column_stack([np.arange(6), h, mh, np.zeros(6)])
    hc, mr = coercivity_remanence(rows)
    assert hc == pytest.approx(0.5 + 0.5 * 0.4 / 1.0) and mr == pytest.approx(0.8)
    hc, mr = coercivity_remanence(rows[:2])
    assert np.isnan(hc) and np.isnan(mr)
    rows2 = rows.copy()
    rows2[:, 1] = [1.0, 0.25, -0.25, -0.5, -1.0, -1.5]  # H = 0 between two steps
    assert coercivity_remanence(rows2)[1] == pytest.approx(0.85)


def test_write_dat_matches_reference_text(golden, tmp_path):
    """scripts/tools.py:20-24: ``f'{int(n)} {hext} {mh} {E/mu0}'`` -- the counter, field and
    polarisation columns of the reference's cube.dat are reproduced as text."""
    gold = (golden / "loop_cube.dat").read_text().splitlines()
    rows = np.loadtxt(golden / "loop_cube.dat")
    rows[:, 3] *= runner.MU0_OUT
    runner.write_dat(tmp_path / "x.dat", rows)
    out = (tmp_path / "x.dat").read_text().splitlines()
    assert len(out) == len(gold)
    for a, b in zip(out, gold):
        fa, fb = a.split(), b.split()
        assert fa[:3] == fb[:3]
        assert float(fa[3]) == pytest.approx(float(fb[3]), rel=1e-15)


def test_initial_states(cube_mesh):
    """scripts/magnetization.py:9-70 getM: mask * state, normalised; non-magnetic nodes 0."""
    X, T, tag = cube_mesh
    krn = O.read_krn_rows((ROOT / "tests" / "golden" / "loop_cube.krn").read_text())
    P = O.Problem(X, T, tag, krn)
    meas = P.meas
    mask = meas > 0
    x0, x1, x2 = X[:, 0], X[:, 1], X[:, 2]
    m = runner.initial_m(X, meas, [0.0, 0.0, 1.0], 0).reshape(-1, 3)
    assert np.array_equal(m, O.initial_m_uniform(P, [0.0, 0.0, 1.0]).reshape(-1, 3))
    s = X.max()
    flower = np.column_stack([x0 * x2 / (10 * s), x1 * x2 / (10 * s), np.ones(len(X))])
    r = np.sqrt(x1 ** 2 + x2 ** 2)
    rc = 0.14 * r.max()
    with np.errstate(divide="ignore", invalid="ignore"):
        vortex = np.column_stack([np.exp(-2 * r / rc), -(x2 / r) * np.sqrt(1 - np.exp(-4 * r * r / rc ** 2)),
                                  (x1 / r) * np.sqrt(1 - np.exp(-4 * r * r / rc ** 2))])
    for sid, ref in ((1, flower), (2, vortex)):
        got = runner.initial_m(X, meas, [0.0, 0.0, 1.0], sid).reshape(-1, 3)
        ok = mask & np.isfinite(ref).all(axis=1)  # the vortex axis r = 0 is 0/0 in the formula
        want = ref[ok] / np.linalg.norm(ref[ok], axis=1, keepdims=True)
        np.testing.assert_allclose(got[ok], want, rtol=1e-13, atol=1e-15)
        assert np.all(got[~mask] == 0)
    for sid in (3, 4):
        got = runner.initial_m(X, meas, [0.0, 0.0, 1.0], sid, seed=5).reshape(-1, 3)
        assert np.allclose(np.linalg.norm(got[mask], axis=1), 1.0) and np.all(got[~mask] == 0)
    assert np.array_equal(runner.initial_m(X, meas, [0, 0, 1], 4, seed=5), runner.initial_m(X, meas, [0, 0, 1], 4, seed=5))
