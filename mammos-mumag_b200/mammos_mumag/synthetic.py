"""Seeded synthetic meshes for the benchmark configurations.

* ``cube_grid(n, L)``: an origin-centred cube of edge ``L`` (nm) split into ``n^3`` cells of
  6 tetrahedra each (Freudenthal/Kuhn split along the main diagonal, positively oriented).
  Coordinates ``x_i = (2i - n) L / (2n)`` are exactly antisymmetric, so only the 8 corners
  sit at the largest radius and the reference's bare-box ("airbox") boundary branch applies
  (``scripts/matrix.py:49-58``).
* ``voronoi_grains``: tet label = nearest of ``g`` seeded grain centres (by centroid); tets
  whose centroid lies within ``gb/2`` of a bisector plane form a grain-boundary phase.
* ``cone_axes``: easy axes drawn uniformly inside a cone about +z.
* ``initial_m``: uniform +z plus a seeded Gaussian perturbation, renormalised.
"""

from __future__ import annotations

import itertools
import math

import numpy as np


def cube_grid(n: int, L: float) -> tuple[np.ndarray, np.ndarray]:
    h2 = L / (2 * n)
    c = (2 * np.arange(n + 1) - n) * h2
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    X = np.column_stack([x.ravel(), y.ravel(), z.ravel()])
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = (i + (n + 1) * (j + (n + 1) * k)).ravel()
    step = np.array([1, n + 1, (n + 1) ** 2])
    tets = []
    for perm in itertools.permutations(range(3)):
        v1 = base + step[perm[0]]
        v2 = v1 + step[perm[1]]
        v3 = base + step.sum()
        tets.append(np.column_stack([base, v1, v2, v3]))
    T = np.concatenate(tets).astype(np.int64)
    P = X[T]
    det = np.einsum("ij,ij->i", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))
    flip = det < 0
    T[flip, 1], T[flip, 2] = T[flip, 2].copy(), T[flip, 1].copy()
    order = np.lexsort((T[:, 0], T.min(axis=1)))
    return X, T[order].astype(np.int32)


def voronoi_grains(X, T, ngrains: int, L: float, rng, gb: float = 2.0) -> np.ndarray:
    """Tags 1..ngrains for grains and ngrains+1 for the boundary phase (if gb > 0)."""
    seeds = rng.uniform(-L / 2, L / 2, size=(ngrains, 3))
    cen = X[T].mean(axis=1)
    d2 = ((cen[:, None, :] - seeds[None, :, :]) ** 2).sum(-1)
    a = d2.argmin(axis=1)
    tag = (a + 1).astype(np.int32)
    if gb > 0 and ngrains > 1:
        da = d2[np.arange(len(a)), a]
        dist = np.full(len(a), np.inf)
        for b in range(ngrains):
            sep = np.linalg.norm(seeds[b] - seeds[a], axis=1)
            with np.errstate(divide="ignore", invalid="ignore"):
                db = (d2[:, b] - da) / (2 * sep)
            db[a == b] = np.inf
            dist = np.minimum(dist, db)
        tag[dist < gb / 2] = ngrains + 1
    return tag


def cone_axes(ngrains: int, cone_deg: float, rng) -> tuple[np.ndarray, np.ndarray]:
    cmin = math.cos(math.radians(cone_deg))
    theta = np.arccos(1 - rng.uniform(size=ngrains) * (1 - cmin))
    phi = 2 * np.pi * rng.uniform(size=ngrains)
    return theta, phi


def initial_m(N: int, rng, sigma: float = 0.01) -> np.ndarray:
    m = np.zeros((N, 3))
    m[:, 2] = 1.0
    m += sigma * rng.standard_normal((N, 3))
    m /= np.linalg.norm(m, axis=1, keepdims=True)
    return m.ravel()


# material of the single-grain and batched configurations: Js=1.61 T, A=7.7e-12 J/m, K1=4.3e6 J/m^3
GRAIN = dict(K1=4.3e6, Js=1.61, A=7.7e-12)
BOUNDARY = dict(K1=0.0, Js=0.5, A=2e-12)


def krn_rows(theta, phi, ngb: int = 0):
    """``.krn`` rows ``theta phi K1 K2 Js A`` for grains (+ one boundary row)."""
    rows = [[float(t), float(p), GRAIN["K1"], 0.0, GRAIN["Js"], GRAIN["A"]] for t, p in zip(theta, phi)]
    if ngb:
        rows.append([0.0, 0.0, BOUNDARY["K1"], 0.0, BOUNDARY["Js"], BOUNDARY["A"]])
    return rows


def single_grain(n: int = 16, L: float = 20.0, seed: int = 0):
    """One cubic grain, easy axis +z (the 20 nm, 16^3 configuration at n=16)."""
    X, T = cube_grid(n, L)
    tag = np.ones(T.shape[0], np.int32)
    rng = np.random.default_rng(seed)
    return X, T, tag, krn_rows([0.0], [0.0]), initial_m(X.shape[0], rng)


def multigrain(n: int = 32, L: float = 80.0, grains: int = 8, cone_deg: float = 15.0, gb: float = 2.0, seed: int = 0):
    """Voronoi multigrain cube with a soft grain-boundary phase (80 nm, 32^3, 8 grains at defaults)."""
    rng = np.random.default_rng(seed)
    X, T = cube_grid(n, L)
    tag = voronoi_grains(X, T, grains, L, rng, gb)
    theta, phi = cone_axes(grains, cone_deg, rng)
    rows = krn_rows(theta, phi, ngb=1 if gb > 0 and grains > 1 else 0)
    present = np.unique(tag)
    rows = [rows[t - 1] for t in present]  # one row per tag present, ascending
    return X, T, tag, rows, initial_m(X.shape[0], rng)
