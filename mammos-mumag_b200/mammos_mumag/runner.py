"""In-process replacement of ``run-escript scripts/loop.py <name>``.

Reads ``<name>.fly``, ``<name>.krn`` and ``<name>.p2`` from the working directory exactly as
the reference's script does (``scripts/tools.py:64-120``, ``scripts/materials.py:12-41``,
``scripts/mapping.py:171-236``), runs the field sweep on the GPU through
``libmumag_b200.so`` and writes the same outputs: ``<name>.dat``
(``scripts/tools.py:20-24``), ``<name>_NNNN.vtu`` snapshots (``scripts/loop.py:103-116``)
and ``<name>_stats.txt`` (``scripts/loop.py:150-172``).
"""

from __future__ import annotations

import configparser
import gc
import inspect
import math
import os
import pathlib

import numpy as np
import scipy.constants

from . import _native, fly, vtu

MU0_OUT = scipy.constants.mu_0


def _normalize3(v):
    s = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return list(v) if s == 0.0 else [v[0] / s, v[1] / s, v[2] / s]


def read_script_params(path) -> dict:
    """``scripts/tools.py:64-120`` (``read_params``) plus the optional ``[b200]`` section
    (``precision = fp64|mixed``, ``dirichlet_rhs = reference|zero``,
    ``mbar = reference|current``) that the reference ignores."""
    cfg = configparser.ConfigParser({
        "mstep": 1.0, "state": "mxyz", "mfinal": -0.8, "hmag_on": 1, "tol_fun": 1e-10,
        "tol_hmag_factor": 1.0, "precond_iter": 10, "iter_max": 1000, "verbose": 1,
    })
    cfg.read(path)
    ist, fld, mnz = cfg["initial state"], cfg["field"], cfg["minimizer"]
    tol_fun = float(mnz["tol_fun"])
    p = dict(
        m=_normalize3([float(ist["mx"]), float(ist["my"]), float(ist["mz"])]),
        state_id={"flower": 1, "vortex": 2, "twisted": 3, "random": 4}.get(ist["state"].lower(), 0),
        hdir=_normalize3([float(fld["hx"]), float(fld["hy"]), float(fld["hz"])]),
        hstart=float(fld["hstart"]), hfinal=float(fld["hfinal"]), hstep=float(fld["hstep"]),
        mstep=float(fld["mstep"]), mfinal=float(fld["mfinal"]),
        hmag_on=int(mnz["hmag_on"]),  # read from [minimizer] as the reference does
        tol_fun=tol_fun, tol_u=tol_fun * float(mnz["tol_hmag_factor"]),
        precond_iter=int(mnz["precond_iter"]),
        precision="fp64", dirichlet_rhs="reference", mbar="reference",
    )
    if cfg.has_section("b200"):
        b = cfg["b200"]
        p["precision"] = b.get("precision", "fp64").strip().lower()
        p["dirichlet_rhs"] = b.get("dirichlet_rhs", "reference").strip().lower()
        p["mbar"] = b.get("mbar", "reference").strip().lower()
    return p


def read_krn_rows(path) -> list[list[float]]:
    return [[float(v) for v in ln.split()] for ln in pathlib.Path(path).read_text().splitlines() if ln.strip()]


def initial_m(X, meas, mdir, state_id=0, seed=0) -> np.ndarray:
    """``scripts/magnetization.py:54-70`` ``getM``: ``normalize(mask * m_state)``; the mask is
    ``meas > 0``.  State 4 (random) uses a seeded NumPy generator instead of escript's."""
    N = X.shape[0]
    x0, x1, x2 = X[:, 0], X[:, 1], X[:, 2]
    if state_id == 1:  # flower
        s = X.max()
        m = np.column_stack([x0 * x2 / (10 * s), x1 * x2 / (10 * s), np.ones(N)])
    elif state_id == 2:  # vortex
        r = np.sqrt(x1 * x1 + x2 * x2)
        rc = 0.14 * r.max()
        rs = np.where(r == 0, 1.0, r)
        w = np.sqrt(1 - np.exp(-4 * r * r / (rc * rc)))
        m = np.column_stack([np.exp(-2 * (r / rc)), -(x2 / rs) * w, (x1 / rs) * w])
    elif state_id == 3:  # twisted
        r = np.sqrt(x1 * x1 + x0 * x0)
        rs = np.where(r == 0, 1.0, r)
        s = X.max()
        pos, neg = (x2 > 0).astype(float), (x2 < 0).astype(float)
        m = np.column_stack([
            x0 * x2 / (10 * s) + 4 * (pos * (-x1 / rs) * (x2 / s) + neg * (x1 / rs) * (-x2 / s)),
            x1 * x2 / (10 * s) + 4 * (pos * (x0 / rs) * (x2 / s) + neg * (-x0 / rs) * (-x2 / s)),
            np.ones(N),
        ])
    elif state_id == 4:  # random
        m = 2.0 * np.random.default_rng(seed).uniform(size=(N, 3)) - 1.0
    else:
        m = np.tile(np.asarray(mdir, dtype=np.float64), (N, 1))
    m = m * (meas > 0)[:, None]
    n = np.linalg.norm(m, axis=1, keepdims=True)
    return (m / np.where(n == 0, 1.0, n)).ravel()


def _memory_mb():
    try:
        import psutil

        return psutil.Process(os.getpid()).memory_info().rss / (1024 * 1024)
    except Exception:  # pragma: no cover
        return float("nan")


def write_dat(path, rows) -> None:
    """``scripts/tools.py:20-24``: ``vtk_number hext mh energy/mu0`` per row."""
    with open(path, "w") as f:
        for c, h, mh, e in rows:
            f.write(f"{int(c)} {float(h)!r} {float(mh)!r} {float(e) / MU0_OUT!r}\n")


def run_loop(workdir, name, m0=None, device=0, grid_ctas=0, block_threads=0, return_steps=False):
    """Run the loop of ``<workdir>/<name>.*`` and write its outputs there.

    ``m0`` (optional, [3N] interleaved, mesh-file order) replaces the ``.p2`` initial state.
    Returns the rows ``[counter, hext, mh, E/mu0]`` (and the per-step solver statistics)."""
    wd = pathlib.Path(workdir)
    par = read_script_params(wd / f"{name}.p2")
    mem_pre = _memory_mb()
    X, T, tag = fly.read_mesh(wd / f"{name}.fly")
    krn = read_krn_rows(wd / f"{name}.krn")
    precision = {"fp64": _native.PREC_FP64, "mixed": _native.PREC_MIXED}[par["precision"]]
    dirichlet = {"reference": 0, "zero": 1}[par["dirichlet_rhs"]]
    mesh = _native.Mesh(X, T, tag, krn, size=1e-9, dirichlet_rhs=dirichlet, precision=precision,
                        device=device, grid_ctas=grid_ctas, block_threads=block_threads)
    try:
        meas, _V = mesh.meas()
        m = initial_m(X, meas, par["m"], par["state_id"]) if m0 is None else np.asarray(m0, np.float64).ravel()
        mesh.set_state(m, None, m)
        mem_post = _memory_mb()
        gc.collect()
        mem_gc = _memory_mb()
        (wd / f"{name}_stats.txt").write_text(inspect.cleandoc(f"""
            Memory before escript2jax: {mem_pre} MB.
            Memory after  escript2jax: {mem_post} MB.
            Memory after garbage collection: {mem_gc} MB.
            """))
        sp = _native.solver_params(hdir=par["hdir"], tol_fun=par["tol_fun"], tol_u=par["tol_u"],
                                   precond_iter=par["precond_iter"], hmag_on=par["hmag_on"],
                                   mbar_mode=1 if par["mbar"] == "current" else 0)
        if grid_ctas == 0 and X.shape[0] > 100_000:
            mesh.autotune(sp)  # large meshes: pick the launch shape by timing

        def snapshot(counter, mm, uu):
            vtu.write_vtu(wd / f"{name}_{counter:04d}.vtu", X, T, tag, {"m": mm, "u": uu})

        rows, steps = mesh.loop(par["hstart"], par["hfinal"], par["hstep"], par["mstep"], par["mfinal"], sp,
                                snapshot=snapshot)
    finally:
        mesh.close()
    write_dat(wd / f"{name}.dat", rows)
    out = rows.copy()
    out[:, 3] /= MU0_OUT
    return (out, steps) if return_steps else out


SCRIPTS = ("loop", "exani", "external", "hmag", "mapping", "materials", "magnetization")


def run_script(script, workdir, name, device=0):
    """The in-process counterpart of ``run-escript scripts/<script>.py <name>`` for the
    scripts this build provides: the loop (:func:`run_loop`), the energy known-answer
    scripts and the material / initial-state dumps (``mammos_mumag.diagnostics``)."""
    if script == "loop":
        return run_loop(workdir, name, device=device)
    if script not in SCRIPTS:
        raise ValueError(f"script {script!r} is not provided (one of {', '.join(SCRIPTS)})")
    from . import diagnostics

    return getattr(diagnostics, f"run_{script}")(workdir, name, device=device)


if __name__ == "__main__":
    import sys

    if len(sys.argv) < 2 or len(sys.argv) > 3:
        sys.exit("usage: python -m mammos_mumag.runner modelname [" + "|".join(SCRIPTS) + "]"
                 "   (in the directory of modelname.*; default loop)")
    run_script(sys.argv[2] if len(sys.argv) == 3 else "loop", ".", sys.argv[1])
