"""ASCII VTK UnstructuredGrid writer for loop snapshots.

Stands in for ``esys.weipa.saveVTK`` as called at
``src/mammos_mumag/scripts/escript_tools.py:26-31``: points in mesh-file order, Tet4 cells
(VTK type 10), point data ``m`` (3 components) and ``u``, cell data ``tags``, numbers in
``%e`` format.
"""

from __future__ import annotations

import numpy as np


def _fmt(a: np.ndarray, ncomp: int) -> str:
    a = np.asarray(a, dtype=np.float64).reshape(-1, ncomp)
    fmt = " ".join(["%e"] * ncomp)
    return "\n".join(fmt % tuple(r) for r in a.tolist()) + "\n"


def write_vtu(path, X, T, tag, point_data: dict, time=0.0, cycle=0, cell_data: dict | None = None) -> None:
    """Point data arrays of N x ncomp values; cell data ``tags`` and, optionally, further
    arrays of E x ncomp values (``cell_data``)."""
    X = np.asarray(X)
    T = np.asarray(T)
    n, e = X.shape[0], T.shape[0]
    out = [
        '<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1">\n<UnstructuredGrid>\n',
        '<FieldData>\n<DataArray Name="TIME" type="Float64" format="ascii" NumberOfTuples="1">\n',
        f"{time:e}\n</DataArray>\n</FieldData>\n<FieldData>\n",
        '<DataArray Name="CYCLE" type="Int32" format="ascii" NumberOfTuples="1">\n',
        f"{cycle}\n</DataArray>\n</FieldData>\n",
        f'<Piece NumberOfPoints="{n}" NumberOfCells="{e}">\n<Points>\n',
        '<DataArray NumberOfComponents="3" type="Float64" format="ascii">\n',
        _fmt(X, 3),
        "</DataArray>\n</Points>\n<Cells>\n",
        '<DataArray Name="connectivity" type="Int32" format="ascii">\n',
        "\n".join(" ".join(map(str, r)) for r in T.tolist()) + "\n",
        '</DataArray>\n<DataArray Name="offsets" type="Int32" format="ascii">\n',
        "\n".join(str(4 * (k + 1)) for k in range(e)) + "\n",
        '</DataArray>\n<DataArray Name="types" type="UInt8" format="ascii">\n',
        "10\n" * e,
        "</DataArray>\n</Cells>\n<PointData>\n",
    ]
    for name, arr in point_data.items():
        arr = np.asarray(arr, dtype=np.float64)
        nc = arr.size // n
        out.append(f'<DataArray Name="{name}" type="Float64" NumberOfComponents="{nc}" format="ascii">\n')
        out.append(_fmt(arr, nc))
        out.append("</DataArray>\n")
    out.append('</PointData>\n<CellData>\n<DataArray Name="tags" type="Float64" NumberOfComponents="1" format="ascii">\n')
    out.append(_fmt(np.asarray(tag, dtype=np.float64), 1))
    out.append("</DataArray>\n")
    for name, arr in (cell_data or {}).items():
        arr = np.asarray(arr, dtype=np.float64)
        nc = arr.size // e
        out.append(f'<DataArray Name="{name}" type="Float64" NumberOfComponents="{nc}" format="ascii">\n')
        out.append(_fmt(arr, nc))
        out.append("</DataArray>\n")
    out.append("</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")
    with open(path, "w") as f:
        f.write("".join(out))


def read_point_data(path, names=("m", "u")) -> dict:
    """Named data arrays (point or cell data) of an ASCII ``.vtu`` written by this module or
    by weipa."""
    text = open(path).read()
    res = {}
    for name in names:
        start = text.index(f'<DataArray Name="{name}"')
        start = text.index(">", start) + 1
        end = text.index("</DataArray>", start)
        res[name] = np.array(text[start:end].split(), dtype=np.float64)
    return res
