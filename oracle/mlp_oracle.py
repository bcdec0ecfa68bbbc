"""NumPy restatement of the learned warm start -- THE ORACLE for the network kernels.

Test infrastructure only (see ``oracle/__init__.py``).  The learned warm start has no
counterpart in the reference: the reference's PCG starts from the previous potential
(``src/mammos_mumag/scripts/solvers.py:221-231``, ``x0=u``).  This module restates what the
library's kernels compute so that the tests can check them:

* ``node_features``  the 16 per-node features over the 1-ring (the node and the nodes it
  shares a tetrahedron with, i.e. its row of the Poisson pattern): m_i, u_i, ring mean of
  m and u, ring max of m and u, then the Jacobi-scaled initial residual ``z = (b - S u)/diag S`` over ``sigma = rms(z)``:
  z_i and its ring mean, max and min;
* ``forward`` / ``backward``  the MLP 16 -> 128 -> 128 -> 128 -> 1 with GELU (tanh form),
  rounding to BF16 where the kernels do (the normalised input, the weights of the three
  hidden layers, the hidden activations) and accumulating in float64;
* ``loss``  mean squared error ``mean((y - t/out_scale)^2)``.

The backward pass is the exact gradient of the unrounded network (BF16 rounding treated as
the identity), which the kernels approximate with BF16 operands and FP32 accumulation.
``backward`` is itself checked against central finite differences in float64
(``tests/test_mlp_oracle.py``).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

NIN = 16
HID = 128
GELU_K0 = 0.7978845608028654  # sqrt(2/pi)
GELU_K1 = 0.044715

# parameter layout of the FP32 master vector (mm_model_get_params)
_SIZES = [("W1", (HID, NIN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("w4", (HID,)), ("b4", (1,))]


def num_params() -> int:
    return sum(int(np.prod(s)) for _, s in _SIZES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in _SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[n], dtype=np.float64).ravel() for n, _ in _SIZES])


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_K0 * (x + GELU_K1 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_K0 * (x + GELU_K1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_K0 * (1.0 + 3.0 * GELU_K1 * x * x)


def forward(p: np.ndarray, fmean, fscale, feats, quantize: bool = True):
    """Network output y (before out_scale) and the cache for ``backward``."""
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    P = unpack(p)
    xn = (np.asarray(feats, np.float32) - np.asarray(fmean, np.float32)) * np.asarray(fscale, np.float32)
    h0 = q(xn)
    z1 = h0 @ q(P["W1"]).T + P["b1"]
    h1 = q(gelu(z1))
    z2 = h1 @ q(P["W2"]).T + P["b2"]
    h2 = q(gelu(z2))
    z3 = h2 @ q(P["W3"]).T + P["b3"]
    h3 = q(gelu(z3))
    y = h3 @ P["w4"] + P["b4"][0]
    return y, (h0, z1, h1, z2, h2, z3, h3)


def loss(y, target, out_scale):
    e = y - np.asarray(target, np.float64) / out_scale
    return float(np.mean(e * e))


def backward(p: np.ndarray, cache, y, target, out_scale) -> np.ndarray:
    """Gradient of ``loss`` w.r.t. the parameter vector (layout of ``unpack``)."""
    P = unpack(p)
    h0, z1, h1, z2, h2, z3, h3 = cache
    n = y.shape[0]
    dy = 2.0 * (y - np.asarray(target, np.float64) / out_scale) / n
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = np.outer(dy, P["w4"]) * gelu_grad(z3)
    g["W3"], g["b3"] = dz3.T @ h2, dz3.sum(0)
    dz2 = (dz3 @ P["W3"]) * gelu_grad(z2)
    g["W2"], g["b2"] = dz2.T @ h1, dz2.sum(0)
    dz1 = (dz2 @ P["W2"]) * gelu_grad(z1)
    g["W1"], g["b1"] = dz1.T @ h0, dz1.sum(0)
    return pack(g)


def node_graph(T: np.ndarray, N: int) -> sp.csr_matrix:
    """Node adjacency of a tetrahedral mesh (all pairs of nodes of a tet, diagonal included):
    the pattern of the Poisson matrix."""
    T = np.asarray(T, np.int64)
    r = np.repeat(T, 4, axis=1).ravel()
    c = np.tile(T, (1, 4)).ravel()
    G = sp.csr_matrix((np.ones(r.size), (r, c)), shape=(N, N))
    G.sum_duplicates()
    return G


def node_features(G: sp.csr_matrix, m: np.ndarray, u: np.ndarray, r0: np.ndarray, diag: np.ndarray):
    """``([N, 16] features, sigma)`` of every node; ``G`` from ``node_graph``, ``m``
    interleaved [3N], ``r0 = b - S u`` the initial residual, ``diag`` the diagonal of S."""
    N = G.shape[0]
    M = np.asarray(m, np.float64).reshape(N, 3)
    u = np.asarray(u, np.float64)
    z = np.asarray(r0, np.float64) / np.asarray(diag, np.float64)
    sig = float(np.sqrt(np.mean(z * z)))
    z = z / sig
    cols = [M[:, 0], M[:, 1], M[:, 2], u, z]
    F = np.zeros((N, NIN))
    for i in range(N):
        ring = G.indices[G.indptr[i]:G.indptr[i + 1]]
        mi = [c[ring] for c in cols]
        F[i, 0:3] = M[i]
        F[i, 3] = u[i]
        F[i, 4:8] = [mi[0].mean(), mi[1].mean(), mi[2].mean(), mi[3].mean()]
        F[i, 8:12] = [mi[0].max(), mi[1].max(), mi[2].max(), mi[3].max()]
        F[i, 12:16] = [z[i], mi[4].mean(), mi[4].max(), mi[4].min()]
    return F, sig
