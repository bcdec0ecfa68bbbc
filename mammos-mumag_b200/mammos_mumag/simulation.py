"""Simulation class (``src/mammos_mumag/simulation.py`` of the reference).

``run_loop`` keeps the reference's contract -- it writes ``<name>.fly``, ``<name>.krn`` and
``<name>.p2`` into ``outdir`` and produces ``<name>.dat``, ``<name>_NNNN.vtu``,
``<name>_stats.txt`` and ``info.json`` there -- but runs the loop in process on the GPU
(``mammos_mumag.runner``) instead of ``run-escript scripts/loop.py <name>``.  Failures raise
``RuntimeError("Simulation has failed. ...")`` as the reference's subprocess wrapper does
(``simulation.py:410-431``).  ``run_exani``, ``run_external``, ``run_hmag`` and
``run_mapping`` run the reference's energy known-answer scripts the same way, and
``run_materials`` / ``run_magnetization`` its VTU dumps (``mammos_mumag.diagnostics``);
``run_store`` (a pickle cache of escript's arrays) raises ``NotImplementedError``.
"""

from __future__ import annotations

import datetime
import json
import pathlib

import mammos_mumag
from mammos_mumag import diagnostics, fly, runner
from mammos_mumag.materials import Materials
from mammos_mumag.parameters import Parameters
from mammos_mumag.tools import check_dir


class Simulation:
    """Holds the mesh path, the materials and the parameters of a run."""

    def __init__(self, material_domain_list=None, mesh_filepath=None, materials_filepath=None,
                 parameters_filepath=None, materials=None, parameters=None):
        self.material_domain_list = material_domain_list
        self.mesh_filepath = pathlib.Path(mesh_filepath) if mesh_filepath is not None else None
        self.materials_filepath = materials_filepath
        self.parameters_filepath = parameters_filepath
        self.materials = materials
        self.parameters = parameters
        if isinstance(self.materials, dict) or isinstance(self.materials, list):
            self.materials = Materials(domains=self.materials)
        if material_domain_list is not None:
            self.materials = Materials(domains=material_domain_list)
        elif materials_filepath is not None:
            self.materials = Materials(filepath=materials_filepath)
        if parameters_filepath is not None:
            self.parameters = Parameters(filepath=parameters_filepath)

    def __repr__(self):
        return f"Simulation(mesh_filepath={self.mesh_filepath!r}, materials={self.materials!r}, parameters={self.parameters!r})"

    def check_attribute(self, *args) -> None:
        for attr in args:
            if getattr(self, attr) is None:
                raise AttributeError(f"Attribute `{attr}` has not been defined yet.")

    def _write_inputs(self, outdir, name, b200: dict | None = None):
        self.check_attribute("mesh_filepath", "materials", "parameters")
        fly.copy_as_fly(self.mesh_filepath, outdir / f"{name}.fly")
        self.materials.write_krn(outdir / f"{name}.krn")
        self.parameters.write_p2(outdir / f"{name}.p2")
        if b200:
            with open(outdir / f"{name}.p2", "a") as f:
                f.write("\n[b200]\n" + "".join(f"{k} = {v}\n" for k, v in b200.items()))

    def run_loop(self, outdir="loop", name="out", m0=None, precision=None, dirichlet_rhs=None, mbar=None,
                 device=0):
        r"""Compute the demagnetisation curve (the reference's ``loop`` script).

        Extra keywords (absent from the reference): ``m0`` an explicit initial
        magnetisation [3N]; ``precision`` ``"fp64"`` (default) or ``"mixed"``;
        ``dirichlet_rhs`` ``"reference"`` (default) or ``"zero"``; ``mbar`` ``"reference"``
        (default, M_inv projects with the initial m) or ``"current"``; ``device``.
        """
        outdir = check_dir(outdir)
        b200 = {k: v for k, v in (("precision", precision), ("dirichlet_rhs", dirichlet_rhs), ("mbar", mbar)) if v}
        self._write_inputs(outdir, name, b200)
        self._run(runner.run_loop, outdir, name, m0=m0, device=device)

    @staticmethod
    def _run(fn, outdir, name, **kw):
        """Run one script replacement in ``outdir``; failures raise as the reference's
        subprocess wrapper does (``simulation.py:410-431``), and ``info.json`` is written as
        its ``run_script`` writes it (``simulation.py:88-113``)."""
        try:
            fn(outdir, name, **kw)
        except Exception as e:
            raise RuntimeError(f"Simulation has failed. Exit with error: \n{e}") from e
        with open(outdir / "info.json", "w") as f:
            json.dump({
                "datetime": datetime.datetime.now(datetime.UTC).astimezone().isoformat(timespec="seconds"),
                "mammos_mumag_version": mammos_mumag.__version__,
            }, f)

    def _write_mesh_krn(self, outdir, name):
        self.check_attribute("mesh_filepath", "materials")
        fly.copy_as_fly(self.mesh_filepath, outdir / f"{name}.fly")
        self.materials.write_krn(outdir / f"{name}.krn")

    def _out_of_scope(self, what):
        raise NotImplementedError(
            f"run_{what} is an escript diagnostic of the reference and is not part of the B200 hysteresis path"
        )

    def run_exani(self, outdir="exani", name="out", device=0):
        """Exchange energy density of the test vortex and anisotropy energy density of the
        uniform state (the reference's ``exani`` script, on the GPU path): writes
        ``<name>.fly``, ``<name>.krn``, ``<name>_vortex.csv`` and ``<name>_uniform.csv``."""
        outdir = check_dir(outdir)
        self._write_mesh_krn(outdir, name)
        self._run(diagnostics.run_exani, outdir, name, device=device)

    def run_external(self, outdir="external", name="out", device=0):
        """Zeeman energy density (the reference's ``external`` script, on the GPU path):
        writes ``<name>.fly``, ``<name>.krn``, ``<name>.p2`` and ``<name>.csv``."""
        outdir = check_dir(outdir)
        self._write_inputs(outdir, name)
        self._run(diagnostics.run_external, outdir, name, device=device)

    def run_hmag(self, outdir="hmag", name="out", device=0):
        """Magnetostatic energy density and field of the uniform +z state (the reference's
        ``hmag`` script, on the GPU path): writes ``<name>.fly``, ``<name>.krn``,
        ``<name>.csv`` and ``<name>_hmag.vtu``."""
        outdir = check_dir(outdir)
        self._write_mesh_krn(outdir, name)
        self._run(diagnostics.run_hmag, outdir, name, device=device)

    def run_magnetization(self, outdir="magnetization", name="out"):
        """The ``.p2`` initial state as ``<name>.0000.vtu`` (the reference's
        ``magnetization`` script; host only): writes ``<name>.fly``, ``<name>.krn``,
        ``<name>.p2`` and the VTU."""
        outdir = check_dir(outdir)
        self._write_inputs(outdir, name)
        self._run(diagnostics.run_magnetization, outdir, name)

    def run_mapping(self, outdir="magnetization", name="out", device=0):
        """Energy checks and the total energy of the initial state (the reference's
        ``mapping`` script, on the GPU path): writes ``<name>.fly``, ``<name>.krn``,
        ``<name>.p2``, ``<name>_{zeeman,exchange,anisotropy,hmag,energy}.csv`` and
        ``<name>_stats.txt``."""
        outdir = check_dir(outdir)
        self._write_inputs(outdir, name)
        self._run(diagnostics.run_mapping, outdir, name, device=device)

    def run_materials(self, outdir="materials", name="out"):
        """The per-element material fields as ``<name>_mat.vtu`` (the reference's
        ``materials`` script; host only): writes ``<name>.fly``, ``<name>.krn`` and the VTU."""
        outdir = check_dir(outdir)
        self._write_mesh_krn(outdir, name)
        self._run(diagnostics.run_materials, outdir, name)

    def run_store(self, outdir="magnetization", name="out"):
        self._out_of_scope("store")
