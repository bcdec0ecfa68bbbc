"""Mesh files shipped with the package (``src/mammos_mumag/mesh.py`` of the reference)."""

import pathlib

_MESH_DIR = pathlib.Path(__file__).parent / "mesh"

CUBE_20_nm = _MESH_DIR / "CUBE_20_nm.npz"
"""Cube with 20 nanometer sides inside a spherical air shell (the reference's
``CUBE_20_nm.fly``, stored compressed; every mesh reader here accepts it)."""
