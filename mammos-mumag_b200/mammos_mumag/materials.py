"""Materials: per-domain magnetic parameters and their ``.krn`` / ``.yaml`` files.

Mirrors ``src/mammos_mumag/materials.py`` of the reference (``MaterialDomain``,
``Materials.read/write_krn/write_yaml/add_domain``).  Quantities are plain floats in SI
units: ``Ms`` in A/m, ``K1``/``K2`` in J/m^3, ``A`` in J/m, angles in radians.  A ``.krn``
line is ``theta phi K1 K2 Js A 1.0 0.0`` with ``Js = mu0 Ms`` in tesla
(``src/mammos_mumag/templates/krn.jinja``); the ``.yaml`` file stores ``Ms`` in tesla too
(``materials.py:183-204`` of the reference).
"""

from __future__ import annotations

import dataclasses
import pathlib

import scipy.constants
import yaml
from jinja2 import Environment, FileSystemLoader
from pydantic import TypeAdapter

from .tools import check_path

MU0 = scipy.constants.mu_0
_TEMPLATES = pathlib.Path(__file__).parent / "templates"


_FLOAT = TypeAdapter(float)


def _value(x, unit: str) -> float:
    """Float value of a number or of a unit-carrying object (astropy-like ``.to``); anything
    else raises ``pydantic.ValidationError``, as the reference's pydantic ``MaterialDomain``
    does (``materials.py:17-60`` of the reference)."""
    if hasattr(x, "to") and hasattr(x, "unit"):
        try:
            return _FLOAT.validate_python(x.to(unit).value)
        except Exception:
            return _FLOAT.validate_python(x.value)
    if hasattr(x, "value") and not isinstance(x, (int, float)):
        return _FLOAT.validate_python(x.value)
    return _FLOAT.validate_python(x)


@dataclasses.dataclass
class MaterialDomain:
    """Uniform material domain (one element tag)."""

    theta: float = 0.0
    """Angle of the anisotropy axis from z, radians."""
    phi: float = 0.0
    """Angle of the anisotropy axis from x, radians."""
    K1: float = 0.0
    """First anisotropy constant, J/m^3."""
    K2: float = 0.0
    """Second anisotropy constant, J/m^3 (carried, unused by the solver)."""
    Ms: float = 0.0
    """Spontaneous magnetisation, A/m."""
    A: float = 0.0
    """Exchange stiffness, J/m."""

    def __post_init__(self):
        self.theta = _FLOAT.validate_python(self.theta)
        self.phi = _FLOAT.validate_python(self.phi)
        self.K1 = _value(self.K1, "J / m3")
        self.K2 = _value(self.K2, "J / m3")
        self.Ms = _value(self.Ms, "A / m")
        self.A = _value(self.A, "J / m")

    @property
    def Js(self) -> float:
        """Spontaneous polarisation mu0*Ms in tesla."""
        return self.Ms * MU0


class Materials:
    """Stores, reads and writes material parameters."""

    def __init__(self, domains=None, filepath=None):
        self.domains: list[MaterialDomain] = [
            d if isinstance(d, MaterialDomain) else MaterialDomain(**d) for d in (domains or [])
        ]
        self.filepath = filepath
        if not self.domains and filepath is not None:
            self.read(filepath)

    def __repr__(self):
        return f"Materials(domains={self.domains!r})"

    def add_domain(self, A, Ms, K1, K2, phi, theta) -> None:
        self.domains.append(MaterialDomain(theta=theta, phi=phi, K1=K1, K2=K2, Ms=Ms, A=A))

    def read(self, fname) -> None:
        fpath = check_path(fname)
        if fpath.suffix == ".yaml":
            self.domains = read_yaml(fpath)
        elif fpath.suffix == ".krn":
            self.domains = read_krn(fpath)
        else:
            raise NotImplementedError(f"{fpath.suffix} materials file is not supported.")

    def krn_rows(self) -> list[list[float]]:
        """The ``.krn`` numbers ``theta phi K1 K2 Js A`` of each domain."""
        return [[d.theta, d.phi, d.K1, d.K2, d.Js, d.A] for d in self.domains]

    def write_krn(self, fname) -> None:
        env = Environment(loader=FileSystemLoader(_TEMPLATES))
        text = env.get_template("krn.jinja").render(domains=self.domains)
        pathlib.Path(fname).write_text(text)

    def write_yaml(self, fname) -> None:
        doms = [
            {"theta": d.theta, "phi": d.phi, "K1": d.K1, "K2": d.K2, "Ms": d.Js, "A": d.A}
            for d in self.domains
        ]
        with open(fname, "w") as f:
            yaml.dump(doms, f)


def read_krn(fname) -> list[MaterialDomain]:
    rows = [ln.split() for ln in pathlib.Path(fname).read_text().splitlines() if ln.strip()]
    return [
        MaterialDomain(theta=float(r[0]), phi=float(r[1]), K1=float(r[2]), K2=float(r[3]),
                       Ms=float(r[4]) / MU0, A=float(r[5]))
        for r in rows
    ]


def read_yaml(fname) -> list[MaterialDomain]:
    """Polarisation under ``Ms`` (what ``write_yaml`` stores, in tesla) or ``Js``."""
    with open(fname) as f:
        doms = yaml.safe_load(f)
    return [
        MaterialDomain(theta=float(d["theta"]), phi=float(d["phi"]), K1=float(d["K1"]), K2=float(d["K2"]),
                       Ms=float(d["Ms"] if "Ms" in d else d["Js"]) / MU0, A=float(d["A"]))
        for d in doms
    ]
