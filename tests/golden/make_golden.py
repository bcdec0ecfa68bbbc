"""Regenerate the golden fixtures in this directory from the reference's test data.

The reference (mammos-mumag 0.7.1) ships its regression goldens as text files under
``tests/data``.  Its own hot path cannot run in this environment (it needs esys-escript
and JAX), so the goldens it recorded are the pins for the oracle and for the CUDA path.
This script reads them as plain text and stores compact copies here:

* ``mammos-mumag_b200/mammos_mumag/mesh/CUBE_20_nm.npz`` -- ``tests/data/cube.fly``
                             (identical to the reference's packaged ``mesh/CUBE_20_nm.fly``;
                             9,698 nodes, 53,275 Tet4, tags 1/2/3): X [N,3] f64 (nm),
                             T [E,4] int32 (0-based), tag [E] int8.  It ships with the package
                             as ``mammos_mumag.mesh.CUBE_20_nm``.
* ``loop_cube.dat``       -- ``tests/data/loop/cube.dat`` verbatim (21 rows of the loop golden).
* ``loop_cube.krn/.p2``   -- the material and parameter files of that loop run, verbatim.
* ``loop_cube_0001.npz``  -- point data ``m`` [N,3] and ``u`` [N] of ``tests/data/loop/cube_0001.vtu``.
* ``energies.json``       -- the energy densities of ``tests/data/{hmag,exani,external,mapping}/*.csv``.
* ``io/``                 -- the reference's material/parameter file fixtures, verbatim.

Usage (needs a checkout of the reference; the fixtures are committed, so tests never need it)::

    python tests/golden/make_golden.py <path of the reference checkout>
"""

import json
import pathlib
import shutil
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def read_fly(path):
    """Parse a finley ``.fly`` text mesh (node lines ``id dof tag x y z``, ``Tet4`` lines
    ``id tag n1 n2 n3 n4`` with 1-based node ids)."""
    lines = pathlib.Path(path).read_text().split("\n")
    nn = int(lines[1].split()[1])
    nodes = np.array([[float(v) for v in ln.split()] for ln in lines[2 : 2 + nn]])
    ids = nodes[:, 0].astype(np.int64)
    assert (ids == np.arange(1, nn + 1)).all(), "node ids must be 1..N"
    ne = int(lines[2 + nn].split()[1])
    el = np.array([[int(v) for v in ln.split()] for ln in lines[3 + nn : 3 + nn + ne]])
    return nodes[:, 3:6], (el[:, 2:6] - 1).astype(np.int32), el[:, 1].astype(np.int8)


def read_vtu_point_data(path, names):
    """Return the ASCII point-data arrays ``names`` of a VTK UnstructuredGrid file."""
    text = pathlib.Path(path).read_text()
    out = {}
    for name in names:
        start = text.index(f'<DataArray Name="{name}"')
        start = text.index(">", start) + 1
        end = text.index("</DataArray>", start)
        out[name] = np.array(text[start:end].split(), dtype=np.float64)
    return out


def read_energy_csv(path):
    rows = pathlib.Path(path).read_text().strip().split("\n")[2:]
    return {r.split(",")[0]: float(r.split(",")[1]) for r in rows}


def main(ref_root):
    data = pathlib.Path(ref_root) / "tests" / "data"
    X, T, tag = read_fly(data / "cube.fly")
    pkg_mesh = HERE.parent.parent / "mammos-mumag_b200" / "mammos_mumag" / "mesh"
    pkg_mesh.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(pkg_mesh / "CUBE_20_nm.npz", X=X, T=T, tag=tag)
    shutil.copyfile(data / "loop" / "cube.dat", HERE / "loop_cube.dat")
    shutil.copyfile(data / "loop" / "cube.krn", HERE / "loop_cube.krn")
    shutil.copyfile(data / "loop" / "cube.p2", HERE / "loop_cube.p2")
    pd = read_vtu_point_data(data / "loop" / "cube_0001.vtu", ["m", "u"])
    np.savez_compressed(
        HERE / "loop_cube_0001.npz", m=pd["m"].reshape(-1, 3), u=pd["u"]
    )
    energies = {
        "hmag": read_energy_csv(data / "hmag" / "cube.csv"),
        "exani_vortex": read_energy_csv(data / "exani" / "cube_vortex.csv"),
        "exani_uniform": read_energy_csv(data / "exani" / "cube_uniform.csv"),
        "external": read_energy_csv(data / "external" / "cube.csv"),
        "mapping": {
            k: read_energy_csv(data / "mapping" / f"cube_{k}.csv")
            for k in ("anisotropy", "energy", "exchange", "hmag", "zeeman")
        },
        "krn": {
            "hmag": (data / "hmag" / "cube.krn").read_text(),
            "exani": (data / "exani" / "cube.krn").read_text(),
            "external": (data / "external" / "cube.krn").read_text(),
            "mapping": (data / "mapping" / "cube.krn").read_text(),
        },
        "p2": {
            "external": (data / "external" / "cube.p2").read_text(),
            "mapping": (data / "mapping" / "cube.p2").read_text(),
        },
    }
    (HERE / "energies.json").write_text(json.dumps(energies, indent=1))
    io_dir = HERE / "io"
    io_dir.mkdir(exist_ok=True)
    for sub in ("materials_files", "parameters_files"):
        for f in (data / sub).iterdir():
            shutil.copyfile(f, io_dir / f.name)
    shutil.copyfile(data / "cube.krn", io_dir / "data_cube.krn")
    shutil.copyfile(data / "cube.p2", io_dir / "data_cube.p2")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
