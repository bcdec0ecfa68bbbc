"""Build libmumag_b200.so in-tree (sm_100a only).

    python mammos-mumag_b200/build.py [--verbose-ptxas]

Compiles csrc/*.cu and csrc/*.cpp with nvcc for ``arch=compute_100a,code=sm_100a`` and links
``mammos_mumag/lib/libmumag_b200.so``.  Objects go to ``_build/`` beside this file.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT = HERE / "mammos_mumag" / "lib" / "libmumag_b200.so"
BUILD = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def compile_one(src: pathlib.Path, verbose_ptxas: bool, defines=(), build_dir=None) -> tuple[pathlib.Path, str]:
    obj = (build_dir or BUILD) / (src.stem + ".o")
    cmd = [
        nvcc(), "-c", str(src), "-o", str(obj), "-O3", "-std=c++17", "-lineinfo", *ARCH,
        "-Xcompiler", "-fPIC,-O3", f"-I{INCLUDE}", f"-I{CSRC}", *[f"-D{d}" for d in defines],
    ]
    if verbose_ptxas and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    return obj, res.stderr


def build(verbose_ptxas: bool = False, quiet: bool = True, out: pathlib.Path | None = None,
          defines=()) -> pathlib.Path:
    """Compile and link; ``out``/``defines`` build a variant library elsewhere."""
    srcs = sources()
    target = pathlib.Path(out) if out else OUT
    build_dir = BUILD if out is None else target.parent / ("_build_" + target.stem)
    stamp = max(p.stat().st_mtime for p in srcs + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h")))
    if target.exists() and target.stat().st_mtime > stamp and not verbose_ptxas and out is None:
        return target
    build_dir.mkdir(parents=True, exist_ok=True)
    target.parent.mkdir(parents=True, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: compile_one(s, verbose_ptxas, defines, build_dir), srcs))
    if verbose_ptxas or not quiet:
        for obj, log in results:
            if log.strip():
                print(f"--- {obj.name}\n{log}", file=sys.stderr)
    tmp = target.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-o", str(tmp), *[str(o) for o, _ in results], *ARCH, "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, target)
    return target


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(verbose_ptxas=a.verbose_ptxas, quiet=False))
