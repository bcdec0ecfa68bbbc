"""The reference's energy diagnostics on the GPU path.

In-process replacements of ``run-escript scripts/<script>.py <name>`` for the three
known-answer scripts of the reference, run in the directory that holds ``<name>.fly``,
``<name>.krn`` (and ``<name>.p2`` for ``external``):

* ``exani`` (``scripts/exani.py:42-89``): exchange energy density of the test vortex and
  anisotropy energy density of the uniform state, from the gradient and analytically;
  writes ``<name>_vortex.csv`` and ``<name>_uniform.csv``;
* ``external`` (``scripts/external.py:52-80``): Zeeman energy density at
  ``mu0 Hext = hstart - hstep``; writes ``<name>.csv``;
* ``hmag`` (``scripts/hmag.py:119-165``): magnetostatic energy density of the uniform +z
  state from the field, from the gradient and analytically (``Js^2 / 6 mu0``); writes
  ``<name>.csv`` and ``<name>_hmag.vtu`` (point data ``m``, ``U``, ``h_nodes``; cell data
  ``tags``, ``h``);
* ``materials`` (``scripts/materials.py:50-72``) and ``magnetization``
  (``scripts/magnetization.py:100-112``): VTU dumps of the per-element material fields and of
  the ``.p2`` initial state (host only: no solve is involved);
* ``mapping`` (``scripts/mapping.py:20-131, 238-295``): the same four energies and the total
  energy of the ``.p2`` initial state at ``mu0 Hext = hstart - hstep``; writes
  ``<name>_{zeeman,exchange,anisotropy,hmag,energy}.csv`` (rows named ``E_jax`` as in the
  reference's tables, the values from this library) and ``<name>_stats.txt``.

The energies from the gradient are evaluations of ``total_eg`` by the library
(``mm_energy_grad``) with the other terms switched off: the exchange + anisotropy energy
is the evaluation at zero field without the magnetostatic term, the Zeeman and
magnetostatic energies are differences of two evaluations.  The field ``h = -grad u`` of
the library's potential and the field energy are formed per element on the host.  CSV text
and analytic values follow the scripts (energies divided by ``scipy.constants.mu_0``,
material constants scaled with ``4e-7 pi``).
"""

from __future__ import annotations

import math
import pathlib

import numpy as np

from . import _native, fly, runner, vtu

MU0_OUT = runner.MU0_OUT  # scripts/tools.py:26-27 (scipy.constants.mu_0)
MU0_SCRIPT = 4e-7 * math.pi  # scripts/materials.py:21, scripts/tools.py:61
SIZE = 1e-9  # scripts/materials.py:13: the length unit of the mesh


def write_csv(path, title: str, rows) -> None:
    """The scripts' ``inspect.cleandoc`` tables: a title line, ``name,value,explanation``
    and one line per value (no trailing newline)."""
    lines = [title, "name,value,explanation"] + [f"{n},{v},{e}" for n, v, e in rows]
    pathlib.Path(path).write_text("\n".join(lines))


def read_csv(path) -> dict:
    """``{name: value}`` of a table written by :func:`write_csv` or by the reference."""
    out = {}
    for ln in pathlib.Path(path).read_text().splitlines()[2:]:
        if ln.strip():
            n, v = ln.split(",")[:2]
            out[n] = float(v)
    return out


def vortex_m(X, meas, V):
    """``xM`` (``scripts/magnetization.py:73-82``): ``m = mask (sin kr, cos kr, 0)`` with
    ``kr = k (x + y)``, ``k = pi / (2 V^(1/3))``; not renormalised.  Returns ``(m [3N], k)``."""
    scale = V ** 0.3333333333333333
    k = 0.5 * math.pi / scale
    kr = k * (X[:, 0] + X[:, 1])
    m = np.stack([np.sin(kr), np.cos(kr), np.zeros_like(kr)], axis=1) * (meas > 0)[:, None]
    return m.ravel(), k


def anisotropy_energy(krn_row, m) -> float:
    """``readAnisotropyEnergy`` (``scripts/tools.py:51-62``): ``-mu0 K1 (m . n)^2`` with the
    first material's axis ``n`` and ``m`` normalised."""
    m = runner._normalize3(m)
    theta, phi, K1 = krn_row[0], krn_row[1], krn_row[2]
    n = (math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta))
    return -MU0_SCRIPT * K1 * (m[0] * n[0] + m[1] * n[1] + m[2] * n[2]) ** 2.0


def element_field(X, T, u):
    """``h = -grad u`` of the P1 potential on every element ([E, 3]) and the element volumes."""
    P = X[T]  # [E, 4, 3]
    J = (P[:, 1:, :] - P[:, :1, :])  # rows: edges from vertex 0
    du = u[T[:, 1:]] - u[T[:, :1]]  # [E, 3]
    grad = np.linalg.solve(J, du[:, :, None])[:, :, 0]
    vol = np.abs(np.linalg.det(J)) / 6.0
    return -grad, vol


def element_js(tag, krn):
    """Js of every element: the ``.krn`` row of its tag (rows in ascending tag order), 0 where
    Js <= 0 (``scripts/materials.py:22-35``)."""
    tags = np.unique(tag)
    js = np.array([krn[i][4] if krn[i][4] > 0 else 0.0 for i in range(len(tags))])
    return js[np.searchsorted(tags, tag)]


def field_energy(X, T, tag, krn, u, m, V) -> float:
    """``integrate(-0.5 h . Js m) / V`` (``scripts/hmag.py:142``): per element the volume times
    ``-0.5 Js h . mean(m at the vertices)``, exact for P1 ``m`` and constant ``h``."""
    h, vol = element_field(X, T, u)
    mbar = np.asarray(m).reshape(-1, 3)[T].mean(axis=1)
    js = element_js(tag, krn)
    return float(np.sum(-0.5 * vol * js * np.einsum("ec,ec->e", h, mbar)) / V)


def _open(wd, name, device):
    X, T, tag = fly.read_mesh(wd / f"{name}.fly")
    krn = runner.read_krn_rows(wd / f"{name}.krn")
    mesh = _native.Mesh(X, T, tag, krn, size=SIZE, device=device)
    return X, T, tag, krn, mesh


def _energy(mesh, m, h, sp) -> float:
    mesh.set_state(m, None, m)
    return mesh.energy_grad(h, sp)[0]


def run_exani(workdir, name, device=0) -> dict:
    """``scripts/exani.py:42-89``: writes ``<name>_vortex.csv`` and ``<name>_uniform.csv``."""
    wd = pathlib.Path(workdir)
    X, T, tag, krn, mesh = _open(wd, name, device)
    try:
        meas, V = mesh.meas()
        off = _native.solver_params(hmag_on=0)
        mv, k = vortex_m(X, meas, V)
        ev = _energy(mesh, mv, 0.0, off) / MU0_OUT
        uniform = [0.0, 0.0, 1.0]
        eu = _energy(mesh, runner.initial_m(X, meas, uniform), 0.0, off) / MU0_OUT
    finally:
        mesh.close()
    A = krn[0][5]
    # scripts/exani.py:60-64 rebinds mu0 to scipy's value before this line
    ev_a = (2 * k * k * MU0_OUT * A / (SIZE * SIZE)) / MU0_OUT
    eu_a = anisotropy_energy(krn[0], uniform) / MU0_OUT
    write_csv(wd / f"{name}_vortex.csv", "Exchange energy density of a vortex on a, b plane.", [
        ("E_gradient", ev, "Energy evaluated from gradient (J/m^3)."),
        ("E_analytic", ev_a, "Energy evaluated analytically (J/m^3)."),
    ])
    write_csv(wd / f"{name}_uniform.csv",
              f"Magnetocrystalline anisotropy energy density of uniformly magnetized sample in direction {uniform}.", [
                  ("E_gradient", eu, "Energy evaluated from gradient (J/m^3)."),
                  ("E_analytic", eu_a, "Energy evaluated analytically (J/m^3)."),
              ])
    return {"vortex": {"E_gradient": ev, "E_analytic": ev_a}, "uniform": {"E_gradient": eu, "E_analytic": eu_a}}


def run_external(workdir, name, device=0) -> dict:
    """``scripts/external.py:52-80``: writes ``<name>.csv``."""
    wd = pathlib.Path(workdir)
    par = runner.read_script_params(wd / f"{name}.p2")
    X, T, tag, krn, mesh = _open(wd, name, device)
    value = par["hstart"] - par["hstep"]  # External.value, scripts/external.py:19
    try:
        meas, _ = mesh.meas()
        m = runner.initial_m(X, meas, par["m"])
        sp = _native.solver_params(hdir=par["hdir"], hmag_on=0)
        eg = (_energy(mesh, m, value, sp) - _energy(mesh, m, 0.0, sp)) / MU0_OUT
    finally:
        mesh.close()
    mdir, hdir, js = par["m"], par["hdir"], krn[0][4]
    ea = -js * (par["hstart"] - par["hstep"]) * (mdir[0] * hdir[0] + mdir[1] * hdir[1] + mdir[2] * hdir[2]) / MU0_OUT
    write_csv(wd / f"{name}.csv", f"Zeeman energy density for an external field of mu_0 Hext {value} (T).", [
        ("E_gradient", eg, "Energy evaluated from gradient (J/m^3)."),
        ("E_analytic", ea, "Energy evaluated analytically (J/m^3)."),
    ])
    return {"E_gradient": eg, "E_analytic": ea, "mu0_Hext": value}


def run_hmag(workdir, name, device=0) -> dict:
    """``scripts/hmag.py:119-165``: writes ``<name>.csv`` and ``<name>_hmag.vtu``."""
    wd = pathlib.Path(workdir)
    X, T, tag, krn, mesh = _open(wd, name, device)
    try:
        meas, V = mesh.meas()
        m = runner.initial_m(X, meas, [0.0, 0.0, 1.0])
        on, off = _native.solver_params(hmag_on=1), _native.solver_params(hmag_on=0)
        e_on = _energy(mesh, m, 0.0, on)
        _, u, g_on = mesh.get_state()
        e_off = _energy(mesh, m, 0.0, off)
        _, _, g_off = mesh.get_state()
    finally:
        mesh.close()
    eg = (e_on - e_off) / MU0_OUT
    ef = field_energy(X, T, tag, krn, u, m, V) / MU0_OUT
    js = krn[0][4]
    ea = (js * js / 6) / MU0_OUT
    write_csv(wd / f"{name}.csv", "Magnetostatic energy density of uniformly magnetized cube.", [
        ("E_field", ef, "Energy density evaluated from field (J/m^3)."),
        ("E_gradient", eg, "Energy density evaluated from gradient (J/m^3)."),
        ("E_analytic", ea, "Energy density evaluated analytically (J/m^3)."),
    ])
    # the magnetostatic part of the gradient, G u, and the nodal field -V G u / meas
    gh = (g_on - g_off).reshape(-1, 3)
    mz = np.where(meas == 0, 1.0, meas)
    h_nodes = -V * gh / mz[:, None]
    h_cells, _ = element_field(X, T, u)
    vtu.write_vtu(wd / f"{name}_hmag.vtu", X, T, tag, {"m": m, "U": u, "h_nodes": h_nodes},
                  cell_data={"h": h_cells})
    return {"E_field": ef, "E_gradient": eg, "E_analytic": ea}


def run_mapping(workdir, name, device=0) -> dict:
    """``scripts/mapping.py:238-295`` with its checks (``:20-131``): writes
    ``<name>_zeeman.csv``, ``<name>_exchange.csv``, ``<name>_anisotropy.csv``,
    ``<name>_hmag.csv``, ``<name>_energy.csv`` and ``<name>_stats.txt``.  The total energy's
    analytic row is the sum of the Zeeman, exchange + anisotropy and magnetostatic energies
    of the checks on the initial state (the reference's table holds that sum)."""
    import time

    wd = pathlib.Path(workdir)
    par = runner.read_script_params(wd / f"{name}.p2")
    t0 = time.perf_counter()
    X, T, tag, krn, mesh = _open(wd, name, device)
    value = par["hstart"] - par["hstep"]  # scripts/mapping.py:26
    try:
        meas, V = mesh.meas()
        m = runner.initial_m(X, meas, par["m"], par["state_id"])
        off = _native.solver_params(hdir=par["hdir"], hmag_on=0)
        on = _native.solver_params(hdir=par["hdir"], hmag_on=1, tol_u=1e-10)  # scripts/mapping.py:107
        e_c = _energy(mesh, m, 0.0, off)  # exchange + anisotropy of the initial state
        e_zee = _energy(mesh, m, value, off) - e_c
        mv, k = vortex_m(X, meas, V)
        e_vortex = _energy(mesh, mv, 0.0, off)
        e_hmag = _energy(mesh, m, 0.0, on) - e_c
        t1 = time.perf_counter()
        full = _native.solver_params(hdir=par["hdir"], hmag_on=par["hmag_on"], tol_u=par["tol_u"])
        e_total = _energy(mesh, m, value, full)
        t2 = time.perf_counter()
    finally:
        mesh.close()
    mdir, hdir, js, A = par["m"], par["hdir"], krn[0][4], krn[0][5]
    uniform = [0.0, 0.0, 1.0]
    rows = {
        "zeeman": (f"Zeeman energy density for an external field of mu_0 Hext {value} (T).", e_zee / MU0_OUT,
                   -js * value * (mdir[0] * hdir[0] + mdir[1] * hdir[1] + mdir[2] * hdir[2]) / MU0_OUT),
        "exchange": ("Exchange energy density of a vortex on a, b plane.", e_vortex / MU0_OUT,
                     (2 * k * k * MU0_OUT * A / (SIZE * SIZE)) / MU0_OUT),
        "anisotropy": ("Magnetocrystalline anisotropy energy density of uniformly magnetized sample in direction "
                       f"{uniform}.", e_c / MU0_OUT, anisotropy_energy(krn[0], uniform) / MU0_OUT),
        "hmag": ("Magnetostatic energy density of uniformly magnetized cube.", e_hmag / MU0_OUT,
                 (js * js / 6) / MU0_OUT),
        "energy": ("Total energy density of uniformly magnetized state.", e_total / MU0_OUT,
                   (e_zee + e_c + e_hmag) / MU0_OUT),
    }
    out = {}
    for key, (title, e_num, e_ana) in rows.items():
        write_csv(wd / f"{name}_{key}.csv", title, [
            ("E_jax", e_num, "Energy evaluated with jax backend (J/m^3)."),
            ("E_analytic", e_ana, "Energy evaluated analytically (J/m^3)."),
        ])
        out[key] = {"E_jax": e_num, "E_analytic": e_ana}
    (wd / f"{name}_stats.txt").write_text("\n".join([
        "MAP FINITE ELEMENT BACKEND TO THE B200 LIBRARY.",
        "Timing and statistics.",
        f"set-up and checks: {t1 - t0}",
        f"elapsed time: {t2 - t1}",
        "function_calls: 1",
    ]))
    return out


def _magnetic_nodes(N, T, tag, krn):
    """``wherePositive(meas)``: nodes of at least one element whose material has Js > 0."""
    mask = np.zeros(N, dtype=bool)
    mask[np.asarray(T)[element_js(tag, krn) > 0].ravel()] = True
    return mask


def run_materials(workdir, name, device=0) -> None:
    """``scripts/materials.py:50-72`` (``Materials.write_vtk``): ``<name>_mat.vtu`` with cell
    data ``u`` (easy axis), ``K`` (= K1, J/m^3), ``Js`` (T) and ``A`` (= mu0 A: the script
    stores A scaled by mu0 / size^2 and writes it times size^2); zero where Js <= 0."""
    wd = pathlib.Path(workdir)
    X, T, tag = fly.read_mesh(wd / f"{name}.fly")
    krn = runner.read_krn_rows(wd / f"{name}.krn")
    tags = np.unique(tag)
    rows = np.zeros((len(tags), 6))  # u (3), K, Js, A
    for i in range(len(tags)):
        theta, phi, K1, _, js, A = krn[i][:6]
        if js > 0:
            rows[i] = [math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta),
                       (MU0_SCRIPT * K1) / MU0_SCRIPT, js, (MU0_SCRIPT * A / (SIZE * SIZE)) * (SIZE * SIZE)]
    per = rows[np.searchsorted(tags, tag)]
    vtu.write_vtu(wd / f"{name}_mat.vtu", X, T, tag, {},
                  cell_data={"u": per[:, 0:3], "K": per[:, 3], "Js": per[:, 4], "A": per[:, 5]})


def run_magnetization(workdir, name, device=0) -> None:
    """``scripts/magnetization.py:100-112``: ``<name>.0000.vtu`` with the ``.p2`` initial state
    (``getM``: uniform, flower, vortex, twisted or random, masked and normalised)."""
    wd = pathlib.Path(workdir)
    par = runner.read_script_params(wd / f"{name}.p2")
    X, T, tag = fly.read_mesh(wd / f"{name}.fly")
    krn = runner.read_krn_rows(wd / f"{name}.krn")
    mask = _magnetic_nodes(len(X), T, tag, krn)
    m = runner.initial_m(X, mask.astype(np.float64), par["m"], par["state_id"])
    vtu.write_vtu(wd / f"{name}.0000.vtu", X, T, tag, {"m": m})
