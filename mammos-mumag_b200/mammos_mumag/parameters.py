"""Simulation parameters and their ``.p2`` / ``.yaml`` files.

Mirrors ``src/mammos_mumag/parameters.py`` of the reference: the same fields and defaults
(``:42-67``), the same ``.p2`` sections ``[mesh] [initial state] [field] [minimizer]``
(``templates/p2.jinja``) and the same reading rules (``:96-167``).
"""

from __future__ import annotations

import configparser
import math
import pathlib

import yaml
from jinja2 import Environment, FileSystemLoader
from pydantic import TypeAdapter

from .tools import check_path

_TEMPLATES = pathlib.Path(__file__).parent / "templates"
_VEC3 = TypeAdapter(list[float])


def _vec3(v, name):
    if hasattr(v, "tolist"):
        v = v.tolist()
    out = _VEC3.validate_python(v)  # raises pydantic.ValidationError for scalars
    if len(out) != 3:
        _VEC3.validate_python(f"{name} must have exactly 3 components")  # ValidationError
    return out


def _normalize(v):
    s = math.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2)
    if s <= 1.0e-13:
        return list(v)
    return [v[0] / s, v[1] / s, v[2] / s]


class Parameters:
    """Simulation parameters (see the reference's ``Parameters`` for their meaning)."""

    _FIELDS = dict(
        size=1.0e-09, scale=0.0, state="", m_vect=None, hmag_on=1, hstart=0.0, hfinal=0.0, hstep=0.0,
        h_vect=None, mstep=1.0, mfinal=-0.8, iter_max=1000, precond_iter=10, tol_fun=1e-10,
        tol_hmag_factor=1.0, tol_u=1e-10, verbose=0,
    )

    def __init__(self, filepath=None, m=None, h=None, **kw):
        unknown = set(kw) - set(self._FIELDS)
        if unknown:
            raise TypeError(f"unknown parameters {sorted(unknown)}")
        for k, v in self._FIELDS.items():
            setattr(self, k, kw.get(k, v))
        self.m_vect = _vec3(self.m_vect if self.m_vect is not None else [0, 0, 0], "m_vect")
        self.h_vect = _vec3(self.h_vect if self.h_vect is not None else [0, 0, 0], "h_vect")
        if m is not None:
            self.m = m
        if h is not None:
            self.h = h
        self.filepath = filepath
        if filepath is not None:
            self.read(filepath)

    def __repr__(self):
        return "Parameters(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in self._FIELDS) + ")"

    @property
    def m(self):
        """Normalised initial magnetisation direction."""
        return _normalize(self.m_vect)

    @m.setter
    def m(self, value):
        self.m_vect = _normalize(_vec3(value, "m"))

    @property
    def h(self):
        """Normalised external field direction."""
        return _normalize(self.h_vect)

    @h.setter
    def h(self, value):
        self.h_vect = _normalize(_vec3(value, "h"))

    def read(self, fname) -> None:
        fpath = check_path(fname)
        if fpath.suffix == ".yaml":
            with open(fpath) as f:
                pars = yaml.safe_load(f)
        elif fpath.suffix == ".p2":
            pars = configparser.ConfigParser()
            pars.read(fpath)
        else:
            raise NotImplementedError(f"{fpath.suffix} materials file is not supported.")
        mesh = pars["mesh"]
        if "size" in mesh:
            self.size = float(mesh["size"])
        if "scale" in mesh:
            self.scale = float(mesh["scale"])
        ist = pars["initial state"]
        if "state" in ist:
            self.state = str(ist["state"])
        self.m = [float(ist["mx"]), float(ist["my"]), float(ist["mz"])]
        fld = pars["field"]
        if "hmag_on" in fld:
            self.hmag_on = int(fld["hmag_on"])
        self.hstart = float(fld["hstart"])
        self.hfinal = float(fld["hfinal"])
        self.hstep = float(fld["hstep"])
        self.h = [float(fld["hx"]), float(fld["hy"]), float(fld["hz"])]
        if "mstep" in fld:
            self.mstep = float(fld["mstep"])
        if "mfinal" in fld:
            self.mfinal = float(fld["mfinal"])
        mnz = pars["minimizer"]
        if "iter_max" in mnz:
            self.iter_max = int(mnz["iter_max"])
        if "precond_iter" in mnz:
            self.precond_iter = int(mnz["precond_iter"])
        if "tol_fun" in mnz:
            self.tol_fun = float(mnz["tol_fun"])
        if "tol_hmag_factor" in mnz:
            self.tol_hmag_factor = float(mnz["tol_hmag_factor"])
        self.tol_u = self.tol_fun * self.tol_hmag_factor
        if "verbose" in mnz:
            self.verbose = int(mnz["verbose"])

    def _render_dict(self):
        d = {k: getattr(self, k) for k in self._FIELDS}
        d.update(mx=self.m[0], my=self.m[1], mz=self.m[2], hx=self.h[0], hy=self.h[1], hz=self.h[2])
        return d

    def write_p2(self, fname) -> None:
        env = Environment(loader=FileSystemLoader(_TEMPLATES))
        pathlib.Path(fname).write_text(env.get_template("p2.jinja").render(self._render_dict()))

    def write_yaml(self, fname) -> None:
        d = {
            "mesh": {"size": self.size, "scale": self.scale},
            "initial state": {"state": self.state, "mx": self.m[0], "my": self.m[1], "mz": self.m[2]},
            "field": {"hmag_on": self.hmag_on, "hstart": self.hstart, "hfinal": self.hfinal, "hstep": self.hstep,
                      "hx": self.h[0], "hy": self.h[1], "hz": self.h[2]},
            "minimizer": {"iter_max": self.iter_max, "tol_fun": self.tol_fun, "tol_hmag_factor": self.tol_hmag_factor,
                          "precond_iter": self.precond_iter, "verbose": self.verbose},
        }
        with open(fname, "w") as f:
            yaml.dump(d, f)
