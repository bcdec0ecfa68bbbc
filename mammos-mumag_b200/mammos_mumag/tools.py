"""Tool functions (``src/mammos_mumag/tools.py`` of the reference)."""

import pathlib


def check_path(fname) -> pathlib.Path:
    """Return the resolved path of an existing file; raise FileNotFoundError otherwise."""
    path = pathlib.Path(fname).resolve()
    if not path.is_file():
        raise FileNotFoundError("File not found.")
    return path


def check_dir(outdir) -> pathlib.Path:
    """Create ``outdir`` (with parents) if needed and return it."""
    outdir = pathlib.Path(outdir)
    outdir.mkdir(exist_ok=True, parents=True)
    return outdir
