"""NumPy/SciPy restatement of mammos-mumag's hysteresis hot path -- THE ORACLE.

This module is test infrastructure.  It exists to check the CUDA path (``libmumag_b200.so``)
and, in ``bench.py``, to time the reference's algorithm on host cores.  Nothing in the
product imports it.

It restates, in plain NumPy/SciPy, what the reference computes through esys-escript
(operator assembly) and JAX (the solver loop).  Neither dependency is importable here
(esys-escript >=5.10,<6 is pinned at ``pyproject.toml:88``; jax is unpinned at
``pyproject.toml:29``).  The algorithms are restated from their call sites:

* materials        ``src/mammos_mumag/scripts/materials.py:12-41``
* meas             ``src/mammos_mumag/scripts/escript_tools.py:13-17``
* operators        ``src/mammos_mumag/scripts/matrix.py:9-74``, ``scripts/trafo.py:4-45``,
                   ``scripts/mapping.py:171-236``
* energy terms     ``src/mammos_mumag/scripts/energies.py:7-99``
* linear solvers   ``src/mammos_mumag/scripts/solvers.py:7-131`` (truncated PCG) and
                   ``:221-231`` (``jax.scipy.sparse.linalg.cg``: standard PCG, stop when
                   ``r.r <= max(tol^2 b.b, atol^2)`` on the unpreconditioned residual)
* minimiser        ``src/mammos_mumag/scripts/minimizers.py:16-190``
* field loop       ``src/mammos_mumag/scripts/loop.py:25-142``
* vector helpers   ``src/mammos_mumag/scripts/jax_tools.py:4-24``
* parameters       ``src/mammos_mumag/scripts/tools.py:64-120``

Pinning: ``tests/test_oracle_golden.py`` checks this module against the reference's own
recorded outputs (``tests/data/loop/cube.dat``, ``cube_0001.vtu``, ``hmag/cube.csv``,
``exani/*.csv``, ``external/cube.csv``, ``mapping/*.csv``), copied as fixtures into
``tests/golden``.  The spherical-shell ("infinity") boundary branch is pinned by those
goldens.  The bare-cube "airbox" branch (``scripts/matrix.py:55-58``) has no golden in
the reference: for that branch the oracle's Dirichlet handling (rows and columns
nullified, diagonal 1, right-hand side not masked) is inferred from escript's constraint
insertion and is *parity unpinned*.

Layout conventions (the reference's): ``m`` is interleaved ``[mx0, my0, mz0, mx1, ...]`` in
mesh-file node order (``scripts/converters.py:36-37``); ``u`` has one value per node.
"""

from __future__ import annotations

import configparser
import math
from dataclasses import dataclass, field

import numpy as np
import scipy.constants
import scipy.sparse as sp

MU0_SCRIPT = 4e-7 * math.pi  # scripts/materials.py:21
MU0_OUT = scipy.constants.mu_0  # scripts/tools.py:26-27 (energy density output)
SQRT_EPS = math.sqrt(np.finfo(np.float64).eps)
QUAD_A = 0.5854101966249685  # 4-point Tet4 rule used by finley for Function(domain)
QUAD_B = 0.1381966011250105

__all__ = [
    "MU0_SCRIPT",
    "MU0_OUT",
    "Problem",
    "read_krn_rows",
    "read_params",
    "initial_m_uniform",
    "normalize_vectors",
    "projection",
    "total_eg",
    "external_g",
    "Stats",
    "update_m",
    "compute_h",
    "alpha_init",
    "dot_magnetizations",
    "pcg",
    "pcg_twolevel",
    "truncated_cg",
    "m_inv",
    "hestenes_stiefel_ncg",
    "compute_mh",
    "run_loop",
    "format_dat",
    "vortex_m",
]


# ----------------------------------------------------------------------------------------
# inputs
# ----------------------------------------------------------------------------------------
def read_krn_rows(text: str) -> list[list[float]]:
    """Rows of a ``.krn`` file: ``theta phi K1 K2 Js A ...`` (``scripts/materials.py:24-34``)."""
    return [[float(v) for v in ln.split()] for ln in text.strip().split("\n") if ln.strip()]


def _normalize3(v):
    """``scripts/tools.py:28-36``: normalise a 3-list, leaving a zero vector unchanged."""
    a, b, c = v
    s = math.sqrt(a * a + b * b + c * c)
    return [a, b, c] if s == 0.0 else [a / s, b / s, c / s]


def read_params(text: str) -> dict:
    """Restates ``scripts/tools.py:64-120`` (``read_params``) on the text of a ``.p2`` file."""
    cfg = configparser.ConfigParser(
        {
            "mstep": 1.0,
            "state": "mxyz",
            "mfinal": -0.8,
            "hmag_on": 1,
            "tol_fun": 1e-10,
            "tol_hmag_factor": 1.0,
            "precond_iter": 10,
            "iter_max": 1000,
            "verbose": 1,
        }
    )
    cfg.read_string(text)
    ist, fld, mnz = cfg["initial state"], cfg["field"], cfg["minimizer"]
    m = _normalize3([float(ist["mx"]), float(ist["my"]), float(ist["mz"])])
    state = ist["state"].lower()
    state_id = {"flower": 1, "vortex": 2, "twisted": 3, "random": 4}.get(state, 0)
    h = _normalize3([float(fld["hx"]), float(fld["hy"]), float(fld["hz"])])
    tol_fun = float(mnz["tol_fun"])
    return dict(
        m=m,
        state_id=state_id,
        hdir=h,
        hstart=float(fld["hstart"]),
        hfinal=float(fld["hfinal"]),
        hstep=float(fld["hstep"]),
        mstep=float(fld["mstep"]),
        mfinal=float(fld["mfinal"]),
        hmag_on=int(mnz["hmag_on"]),  # read from [minimizer] (scripts/tools.py:106)
        tol_fun=tol_fun,
        tol_u=tol_fun * float(mnz["tol_hmag_factor"]),  # scripts/tools.py:111
        precond_iter=int(mnz["precond_iter"]),
        iter_max=int(mnz["iter_max"]),
    )


# ----------------------------------------------------------------------------------------
# operators (what escript/finley assembles)
# ----------------------------------------------------------------------------------------
def _where_zero(arg: np.ndarray) -> np.ndarray:
    """escript ``whereZero(arg)`` with its default ``tol = sqrt(eps) * Lsup(arg)``."""
    tol = SQRT_EPS * np.abs(arg).max()
    return np.abs(arg) <= tol


def _shell_tensor(xq: np.ndarray, R: float, Rinf: float) -> np.ndarray:
    """``scripts/trafo.py:24-45`` ``get_T3D`` at points ``xq[...,3]``."""
    x = np.linalg.norm(xq, axis=-1)
    a2 = R * (Rinf - R)
    ax = Rinf / x
    a2x2 = a2 / (x * x)
    f = ax * (2 - ax) / (ax - 1) ** 2
    xh = xq / x[..., None]
    k = np.empty(xq.shape[:-1] + (3, 3))
    for i in range(3):
        k[..., i, i] = a2x2 * (1 + f * (1 - xh[..., i] ** 2))
    for i, j in ((0, 1), (0, 2), (1, 2)):
        k[..., i, j] = -a2x2 * (f * xh[..., i] * xh[..., j])
        k[..., j, i] = k[..., i, j]
    return k


@dataclass
class Problem:
    """Assembled operators of one mesh, in the reference's layout.

    ``X`` [N,3] node coordinates (nm), ``T`` [E,4] 0-based tets, ``tag`` [E] element tags,
    ``krn`` one ``.krn`` row per element tag in ascending tag order.
    ``dirichlet_rhs``: ``"reference"`` keeps the right-hand side on Dirichlet nodes (what
    escript's constraint insertion gives the reference, ``u_B = b_B``); ``"zero"`` sets it 0.
    """

    X: np.ndarray
    T: np.ndarray
    tag: np.ndarray
    krn: list
    size: float = 1e-9
    dirichlet_rhs: str = "reference"
    # filled by __post_init__
    N: int = field(init=False)
    E: int = field(init=False)

    def __post_init__(self):
        X = np.asarray(self.X, dtype=np.float64)
        T = np.asarray(self.T, dtype=np.int64)
        tag = np.asarray(self.tag)
        self.X, self.T, self.tag = X, T, tag
        N, E = X.shape[0], T.shape[0]
        self.N, self.E = N, E
        tags = sorted(np.unique(tag).tolist())
        self.tags = tags
        if len(self.krn) < len(tags):
            raise ValueError(f".krn has {len(self.krn)} rows for {len(tags)} element tags")
        # --- materials, scripts/materials.py:17-41
        Js_t, K_t, A_t = np.zeros(len(tags)), np.zeros(len(tags)), np.zeros(len(tags))
        u_t = np.zeros((len(tags), 3))
        for i, _t in enumerate(tags):
            row = self.krn[i]
            theta, phi, js = row[0], row[1], row[4]
            if js > 0:
                u_t[i] = [math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta)]
                K_t[i] = MU0_SCRIPT * row[2]
                Js_t[i] = js
                A_t[i] = MU0_SCRIPT * row[5] / (self.size * self.size)
        tidx = np.searchsorted(np.array(tags), tag)
        self.tag_index = tidx
        Js, K, A, uax = Js_t[tidx], K_t[tidx], A_t[tidx], u_t[tidx]
        self.Js_e, self.K_e, self.A_e, self.u_e = Js, K, A, uax
        # --- geometry: P1 gradients and volumes
        P = X[T]
        Dm = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2)
        vol = np.abs(np.linalg.det(Dm)) / 6.0
        Inv = np.linalg.inv(Dm)
        G = np.concatenate([-Inv.sum(1, keepdims=True), Inv], axis=1)  # [E,4,3] grad N_a
        self.vol, self.G = vol, G
        V = float(vol[Js > 0].sum())  # scripts/materials.py:36-37
        if not V > 0:
            raise ValueError("no magnetic material (every Js <= 0)")
        self.V = V
        meas = np.zeros(N)
        np.add.at(meas, T, np.repeat((Js * vol / 4.0)[:, None], 4, 1))  # escript_tools.py:13-17
        self.meas = meas
        self.mask = meas > 0

        rr = np.repeat(T, 4, axis=1).ravel()
        cc = np.tile(T, (1, 4)).ravel()

        def asm(Kloc):
            return sp.csr_matrix((Kloc.ravel(), (rr, cc)), shape=(N, N))

        # --- exchange + anisotropy, scripts/matrix.py:37-47 (consistent mass for D term)
        lap = np.einsum("eic,ejc->eij", G, G) * vol[:, None, None]
        SA = asm(lap * (2.0 * A / V)[:, None, None])
        mass = np.where(np.eye(4)[None] > 0, 2.0, 1.0) * (vol / 20.0)[:, None, None]
        mk = mass * (-2.0 * K / V)[:, None, None]  # [E,4,4]
        # 3N x 3N interleaved: row 3i+p, col 3j+q.  One N x N block per (p, q), each entry
        # the element sum of mk_ab u_p u_q in element order, placed by a Kronecker product
        # (the blocks' stored entries do not overlap); assembled block by block so that the
        # transient COO arrays stay N x N sized on large meshes.
        Kani = None
        for p in range(3):
            for q in range(3):
                unit = sp.csr_matrix(([1.0], ([p], [q])), shape=(3, 3))
                blk = sp.kron(asm(mk * (uax[:, p] * uax[:, q])[:, None, None]), unit, format="csr")
                Kani = blk if Kani is None else Kani + blk
        Cex = sp.kron(SA, sp.eye(3), format="csr")
        self.C = (Cex + Kani).tocsr()
        self.C.sum_duplicates()
        Dex = np.repeat(SA.diagonal(), 3)
        self.D = np.where(np.repeat(meas, 3) == 0, 1.0, Dex)  # scripts/mapping.py:207-209
        self.SA = SA
        # --- divergence / gradient operators, scripts/matrix.py:9-35
        w = (Js * vol / 4.0)[:, None]
        self.dk = [asm(np.repeat((G[:, :, c] * w)[:, :, None], 4, 2)) for c in range(3)]
        self.gk = [(d.T / V).tocsr() for d in self.dk]
        # --- Poisson with boundary treatment, scripts/matrix.py:49-74, trafo.py
        rn = np.linalg.norm(X, axis=1)
        Rinf = rn.max()
        bmask = _where_zero(rn - Rinf)
        self.airbox = abs(int(bmask.sum()) - 8) < 1e-8
        if self.airbox:
            bm = np.zeros(N, dtype=bool)
            for c in range(3):
                xe = X[:, c].max()
                bm |= _where_zero(X[:, c] + xe) | _where_zero(X[:, c] - xe)
            bmask = bm
            kbar = np.broadcast_to(np.eye(3), (E, 3, 3))
        else:
            if len(tags) < 2:
                raise ValueError("shell boundary needs at least two element tags")
            nodes2 = np.unique(T[tag == tags[-2]])
            R = float(rn[nodes2].max())
            Bq = np.full((4, 4), QUAD_B) + np.eye(4) * (QUAD_A - QUAD_B)
            last = tag == tags[-1]
            xq = np.einsum("qi,eic->eqc", Bq, P[last])
            kbar = np.broadcast_to(np.eye(3), (E, 3, 3)).copy()
            kbar[last] = _shell_tensor(xq, R, Rinf).mean(axis=1)
            self.R = R
        self.Rinf = Rinf
        self.bnd = bmask
        Sfull = asm(np.einsum("eia,eab,ejb->eij", G, kbar, G) * vol[:, None, None])
        keep = sp.diags((~bmask).astype(np.float64))
        self.S = (keep @ Sfull @ keep + sp.diags(bmask.astype(np.float64))).tocsr()
        self.S.sum_duplicates()
        self.diagS = self.S.diagonal().copy()

    # b = dx m_x + dy m_y + dz m_z  (scripts/energies.py:43)
    def divergence(self, m):
        b = self.dk[0] @ m[0::3] + self.dk[1] @ m[1::3] + self.dk[2] @ m[2::3]
        if self.dirichlet_rhs == "zero":
            b = np.where(self.bnd, 0.0, b)
        return b


# ----------------------------------------------------------------------------------------
# vector helpers, scripts/jax_tools.py:4-24 and scripts/energies.py:61-65
# ----------------------------------------------------------------------------------------
def normalize_vectors(m):
    v = m.reshape(-1, 3)
    n = np.linalg.norm(v, axis=1, keepdims=True)
    return (v / np.where(n == 0, 1.0, n)).reshape(-1)


def update_m(m, step, d):
    return normalize_vectors(m + step * d)


def projection(m, g):
    a = m.reshape(-1, 3)
    b = g.reshape(-1, 3)
    return np.cross(a, np.cross(b, a)).ravel()


def dot_magnetizations(a, b):
    return np.sum(a.reshape(-1, 3) * b.reshape(-1, 3), axis=1, keepdims=True)


# ----------------------------------------------------------------------------------------
# linear solvers
# ----------------------------------------------------------------------------------------
def pcg(A, D, b, x0, tol, atol=0.0, maxiter=10000):
    """``jax.scipy.sparse.linalg.cg`` with ``M = x * (1/D)`` as called at ``scripts/solvers.py:221-231``.

    Returns ``(x, iterations)``."""
    invD = 1.0 / D
    bs = b @ b
    atol2 = max(tol * tol * bs, atol * atol)
    x = x0.copy()
    r = b - A @ x
    z = r * invD
    p = z.copy()
    gamma = r @ z
    k = 0
    while (r @ r) > atol2 and k < maxiter:
        Ap = A @ p
        alpha = gamma / (p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = r * invD
        gamma_ = r @ z
        beta = gamma_ / gamma
        p = z + beta * p
        gamma = gamma_
        k += 1
    return x, k


def pcg_twolevel(A, D, b, x0, tol, box, atol=0.0, maxiter=10000):
    """PCG with the CUDA path's optional two-level additive preconditioner (no counterpart
    in the reference, whose ``scripts/solvers.py:221-231`` uses Jacobi):
    ``z = r / D + P Ac^-1 P^T r`` with ``P[i, box[i]] = 1`` (``box[i] = -1``: no box) and
    ``Ac = P^T A P``.  Same stop rule as ``pcg`` (the reference's).  Returns ``(x, iterations)``."""
    box = np.asarray(box)
    nc = int(box.max()) + 1
    rows = np.nonzero(box >= 0)[0]
    P = sp.csr_matrix((np.ones(len(rows)), (rows, box[rows])), shape=(A.shape[0], nc))
    Ac = (P.T @ A @ P).toarray()
    Ainv = np.linalg.inv(Ac)
    invD = 1.0 / D

    def prec(r):
        return r * invD + P @ (Ainv @ (P.T @ r))

    bs = b @ b
    atol2 = max(tol * tol * bs, atol * atol)
    x = x0.copy()
    r = b - A @ x
    z = prec(r)
    p = z.copy()
    gamma = r @ z
    k = 0
    while (r @ r) > atol2 and k < maxiter:
        Ap = A @ p
        alpha = gamma / (p @ Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = prec(r)
        gamma_ = r @ z
        p = z + (gamma_ / gamma) * p
        gamma = gamma_
        k += 1
    return x, k


def truncated_cg(Bk, grad_fk, Dk, max_iter):
    """``scripts/solvers.py:7-131``: solve ``Bk p ~ -grad_fk`` by diagonal-PCG, stopping at
    negative curvature or ``|r| <= min(0.5, sqrt|g| |g|)``; an all-zero result falls back to
    ``-grad_fk``.  Returns ``(p, iterations)``."""
    norm_grad = np.linalg.norm(grad_fk)
    eps_k = min(0.5, math.sqrt(norm_grad) * norm_grad)
    p = np.zeros_like(grad_fk)
    r = grad_fk.copy()
    z = r / Dk
    d = -z
    i = 0
    while i < max_iter:
        Bd = Bk(d)
        denom = d @ Bd
        neg = denom <= 0.0
        rz = r @ z
        alpha = 0.0 if neg else rz / denom
        p_new = p + alpha * d
        r_new = r + alpha * Bd
        z_new = r_new / Dk
        conv = np.linalg.norm(r_new) <= eps_k
        i += 1
        if neg:
            break
        p, r, z = p_new, r_new, z_new
        if conv:
            break
        beta = (r_new @ z_new) / (rz + 1e-16)
        d = -z_new + beta * d
    if np.all(p == 0):
        return -grad_fk, i
    return p, i


# ----------------------------------------------------------------------------------------
# energy + gradient, scripts/energies.py:7-99
# ----------------------------------------------------------------------------------------
@dataclass
class Stats:
    evals: int = 0
    pcg_iters: int = 0
    ncg_iters: int = 0
    ls_shrinks: int = 0
    minv_iters: int = 0


def external_g(P: Problem, h, hdir):
    return np.stack([(-h * hdir[c] / P.V) * P.meas for c in range(3)], axis=1).ravel()


def total_eg(P: Problem, m, h, hdir, u0, tol_u, hmag_on=1, stats: Stats | None = None):
    """Returns ``(E, projected gradient, u, full gradient)``."""
    gz = external_g(P, h, hdir)
    energy = m @ gz
    gradient = gz.copy()
    gc = P.C @ m
    energy += 0.5 * (m @ gc)
    gradient += gc
    if hmag_on > 0:
        b = P.divergence(m)
        u, k = pcg(P.S, P.diagS, b, u0, tol_u)
        gh = np.stack([P.gk[0] @ u, P.gk[1] @ u, P.gk[2] @ u], axis=1).ravel()
        energy += 0.5 * (m @ gh)
        gradient += gh
        if stats is not None:
            stats.pcg_iters += k
    else:
        u = u0
    if stats is not None:
        stats.evals += 1
    return energy, projection(m, gradient), u, gradient


def m_inv(P: Problem, g, gradF, mbar, precond_iter, stats: Stats | None = None):
    """``scripts/loop.py:40-55``: truncated PCG on ``A v = mbar x ((C v) x mbar) - (mbar.gradF) v``.

    ``mbar`` is the *initial* magnetisation in the reference (a module global captured
    at trace time), not the current iterate."""
    md = dot_magnetizations(mbar, gradF)

    def A(v):
        return projection(mbar, P.C @ v) - (md * v.reshape(-1, 3)).ravel()

    p, it = truncated_cg(A, -g, P.D, precond_iter)
    if stats is not None:
        stats.minv_iters += it
    return p


# ----------------------------------------------------------------------------------------
# minimiser, scripts/minimizers.py:16-190
# ----------------------------------------------------------------------------------------
def compute_h(x, d):
    t1 = 2.0 * SQRT_EPS * (1.0 + np.linalg.norm(x)) / np.linalg.norm(d)
    t2 = SQRT_EPS / np.abs(d).max()
    return t1 if t1 < t2 else t2


def alpha_init(f0, f, g, d, g1, h, c=0.1, o=0.99):
    gd = g @ d
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        t1 = -h * (gd / ((g1 @ d) - gd))
        t1 = c * abs(t1) if t1 < 0 else t1
        t2 = 2.0 * (f - f0) / gd
    t2 = 1.0e30 if t2 < 0 else t2
    return t1 if t1 < o * t2 else t2


def hestenes_stiefel_ncg(P, x, h, hdir, u, gradF, mbar, par, stats: Stats):
    """One field step: ``scripts/minimizers.py:140-190`` with ``func = total_eg``,
    ``update_x = update_m``, ``M_inv`` from ``scripts/loop.py:40-55``.

    Returns ``(f, x, k, u, gradF)``."""
    tol, tol_u, piter, hm = par["tol_fun"], par["tol_u"], par["precond_iter"], par["hmag_on"]
    iter_max = par.get("max_ncg_iter", 100000)  # scripts/minimizers.py:142

    def func(xx, uu):
        return total_eg(P, xx, h, hdir, uu, tol_u, hm, stats)

    f0 = np.finfo(np.float64).max
    f, g, u, gradF = func(x, u)
    d = -m_inv(P, g, gradF, mbar, piter, stats)
    k = 1
    x0 = x
    sqrt_tol, cbrt_tol = math.sqrt(tol), np.cbrt(tol)
    while True:
        a = (f0 - f) > tol * (1 + abs(f))
        b = np.abs(x0 - x).max() > sqrt_tol * (1 + np.abs(x).max())
        c = np.abs(g).max() > cbrt_tol * (1 + abs(f))
        if not ((a or b or c) and k < iter_max):
            break
        if d @ g > -0.001 * np.linalg.norm(d) * np.linalg.norm(g):
            d = -g
        # --- line search, scripts/minimizers.py:92-137
        hh = compute_h(x, d)
        x1 = update_m(x, hh, d)
        f1, g1, u, gradF = func(x1, u)
        alpha = alpha_init(f0, f, g, d, g1, hh)
        gd = g @ d
        x1 = update_m(x, alpha, d)
        f1, g1, u, gradF = func(x1, u)
        gd1 = g1 @ d
        i = 0
        eps_k = 1e-6 * abs(f)
        while True:
            wolfe = ((2 * 0.1 - 1) * gd >= gd1) and (f1 <= f + eps_k)
            if wolfe or (f1 <= f + 1e-4 * alpha * gd) or i > 20:
                break
            alpha *= 0.5
            x1 = update_m(x, alpha, d)
            f1, g1, u, gradF = func(x1, u)
            gd1 = g1 @ d
            i += 1
            stats.ls_shrinks += 1
        # --- direction update
        z1 = m_inv(P, g1, gradF, mbar, piter, stats)
        y = g1 - g
        beta = max((y @ z1) / (y @ d), 0.0)
        d = -z1 + beta * d
        if d @ g > -0.001 * np.linalg.norm(d) * np.linalg.norm(g):
            d = -z1
        k += 1
        x0, f0, x, f, g = x, f, x1, f1, g1
    stats.ncg_iters += k
    return f, x, k, u, gradF


def compute_mh(P: Problem, m, hdir):
    """``scripts/loop.py:25-38``."""
    return ((hdir[0] * m[0::3] + hdir[1] * m[1::3] + hdir[2] * m[2::3]) @ P.meas) / P.V


def initial_m_uniform(P: Problem, mdir):
    """``scripts/magnetization.py:54-70`` (state 0): ``normalize(mask * v)``."""
    m = np.zeros((P.N, 3))
    m[P.mask] = mdir
    return normalize_vectors(m.ravel())


def vortex_m(P: Problem):
    """``scripts/magnetization.py:73-82`` ``xM``: the exchange test vortex and its wave number."""
    scale = P.V ** 0.3333333333333333
    k = 0.5 * math.pi / scale
    kr = k * (P.X[:, 0] + P.X[:, 1])
    m = np.stack([np.sin(kr), np.cos(kr), np.zeros_like(kr)], axis=1) * P.mask[:, None]
    return m.ravel(), k


def run_loop(P: Problem, par: dict, m0=None, mbar_mode="reference", max_steps=None, snapshot=None):
    """``scripts/loop.py:71-142``: the field sweep.

    Returns ``(rows, per_step_stats)``; ``rows`` are ``[counter, hext, mh, E]`` with E in
    the reference's internal units (divide by ``MU0_OUT`` for J/m^3).  ``snapshot(counter,
    m, u)`` is called where the reference writes ``<name>_<counter>.vtu``."""
    if m0 is None:
        m0 = initial_m_uniform(P, par["m"])
    m = np.asarray(m0, dtype=np.float64).copy()
    hdir = par["hdir"]
    hstart, hfinal, hstep = par["hstart"], par["hfinal"], par["hstep"]
    mstep, mfinal = par["mstep"], par["mfinal"]
    nmax = int(abs(hfinal - hstart) / abs(hstep)) + 1
    if max_steps is not None:
        nmax = min(nmax, max_steps)
    u = np.zeros(P.N)
    gradF = np.zeros(3 * P.N)
    mh = np.finfo(np.float64).max
    last_saved = mh
    counter = 0
    hext = hstart
    rows, step_stats = [], []
    idx = 0
    while mh > mfinal and idx < nmax:
        st = Stats()
        mbar = m0 if mbar_mode == "reference" else m
        e, m, _k, u, gradF = hestenes_stiefel_ncg(P, m, hext, hdir, u, gradF, mbar, par, st)
        mh = compute_mh(P, m, hdir)
        if (last_saved - mh) > mstep:
            counter += 1
            last_saved = mh
            if snapshot is not None:
                snapshot(counter, m, u)
        rows.append([counter, hext, mh, e])
        step_stats.append(st)
        hext = hext + hstep
        idx += 1
    return np.array(rows), step_stats


def format_dat(rows) -> str:
    """``scripts/tools.py:20-24`` ``write_mh``."""
    return "".join(
        f"{int(c)} {float(h)!r} {float(mh)!r} {float(e) / MU0_OUT!r}\n" for c, h, mh, e in rows
    )
