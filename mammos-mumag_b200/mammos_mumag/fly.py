"""Reader and writer of finley ``.fly`` text meshes (the reference's mesh input,
``src/mammos_mumag/scripts/mesh.py:9-15`` reads them with ``esys.finley.ReadMesh``).

Layout: a name line; ``3D-nodes N``; N lines ``id dof tag x y z``; ``Tet4 E``; E lines
``id tag n1 n2 n3 n4`` (node ids); then the empty face/contact/point sections and ``Tags``.
Node ids are mapped to 0-based indices in node-line order, which is also the DOF order of
the reference's arrays (``scripts/converters.py:36-37``).  A compressed ``.npz`` with arrays
``X``, ``T`` (0-based) and ``tag`` is accepted wherever a ``.fly`` path is.
"""

from __future__ import annotations

import pathlib

import numpy as np


def read_mesh(path) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Return ``X`` [N,3] float64, ``T`` [E,4] int32 (0-based), ``tag`` [E] int32."""
    path = pathlib.Path(path)
    if path.suffix == ".npz":
        z = np.load(path)
        return (np.ascontiguousarray(z["X"], np.float64), np.ascontiguousarray(z["T"], np.int32),
                np.ascontiguousarray(z["tag"], np.int32))
    with open(path) as f:
        f.readline()  # mesh name
        hdr = f.readline().split()
        if len(hdr) != 2 or not hdr[0].endswith("nodes"):
            raise ValueError(f"{path}: expected '<dim>D-nodes N', got {' '.join(hdr)!r}")
        nn = int(hdr[1])
        nodes = np.array(" ".join(f.readline() for _ in range(nn)).split(), dtype=np.float64).reshape(nn, 6)
        hdr = f.readline().split()
        if len(hdr) != 2 or hdr[0] != "Tet4":
            raise ValueError(f"{path}: only Tet4 volume elements are supported, got {' '.join(hdr)!r}")
        ne = int(hdr[1])
        el = np.array(" ".join(f.readline() for _ in range(ne)).split(), dtype=np.int64).reshape(ne, 6)
    ids = nodes[:, 0].astype(np.int64)
    if nn == 0 or ne == 0 or ids.min() < 0:
        raise ValueError(f"{path}: needs nodes and Tet4 elements with non-negative node ids")
    ref = el[:, 2:6]
    if ref.min() < 0 or ref.max() > ids.max():
        raise ValueError(f"{path}: element references an undefined node id")
    lookup = np.full(ids.max() + 1, -1, dtype=np.int64)
    lookup[ids] = np.arange(nn)
    T = lookup[ref]
    if (T < 0).any():
        raise ValueError(f"{path}: element references an undefined node id")
    return np.ascontiguousarray(nodes[:, 3:6]), T.astype(np.int32), el[:, 1].astype(np.int32)


def write_mesh(path, X, T, tag, name="Mesh") -> None:
    """Write a finley ``.fly`` text mesh (1-based ids)."""
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.int64)
    tag = np.asarray(tag, dtype=np.int64)
    n, e = X.shape[0], T.shape[0]
    ids = np.arange(1, n + 1)
    with open(path, "w") as f:
        f.write(f"{name}\n3D-nodes {n}\n")
        node = np.column_stack([ids, ids, np.zeros(n, np.int64)])
        f.write("".join(f"{a} {b} {c} {x:.16E} {y:.16E} {z:.16E}\n" for (a, b, c), (x, y, z) in zip(node.tolist(), X.tolist())))
        f.write(f"Tet4 {e}\n")
        el = np.column_stack([np.arange(1, e + 1), tag, T + 1])
        f.write("".join(" ".join(map(str, r)) + "\n" for r in el.tolist()))
        f.write("Tri3 0\nTri3_Contact 0\nPoint1 0\nTags\n")


def copy_as_fly(src, dst) -> None:
    """Copy a mesh to ``dst`` as ``.fly`` text (``.npz`` inputs are converted)."""
    src = pathlib.Path(src)
    if src.suffix == ".npz":
        write_mesh(dst, *read_mesh(src))
    else:
        pathlib.Path(dst).write_bytes(src.read_bytes())
