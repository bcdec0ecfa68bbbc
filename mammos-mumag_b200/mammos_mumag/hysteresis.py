"""Hysteresis front end (``src/mammos_mumag/hysteresis.py`` of the reference).

``run`` builds the same three-domain simulation (magnet + two non-magnetic domains) with
the same parameters (``hysteresis.py:96-110``) and returns a ``Result``.  Without the
``mammos_entity``/``mammos_units`` packages, quantities are plain floats / NumPy arrays in SI
units: ``Ms`` [A/m], ``A`` [J/m], ``K1`` [J/m^3], fields [A/m]; unit-carrying objects with an
astropy-like ``.to(unit)`` are converted.  Plotting (matplotlib / pyvista) is not provided.
"""

from __future__ import annotations

import dataclasses
import pathlib

import numpy as np
import pandas as pd
import scipy.constants

from mammos_mumag.materials import Materials, _value
from mammos_mumag.parameters import Parameters
from mammos_mumag.simulation import Simulation

MU0 = scipy.constants.mu_0


def run(Ms, A, K1, mesh_filepath, hstart, hfinal, hstep=None, hnsteps: int = 20, outdir="hystloop", **loop_kw):
    """Run a hysteresis loop; fields in A/m.  ``loop_kw`` go to ``Simulation.run_loop``."""
    hs, hf = _value(hstart, "A / m"), _value(hfinal, "A / m")
    hp = (hf - hs) / hnsteps if hstep is None else _value(hstep, "A / m")
    sim = Simulation(
        mesh_filepath=mesh_filepath,
        materials=Materials(domains=[
            {"theta": 0, "phi": 0.0, "K1": K1, "K2": 0.0, "Ms": Ms, "A": A},
            {"theta": 0.0, "phi": 0.0, "K1": 0.0, "K2": 0.0, "Ms": 0.0, "A": 0.0},
            {"theta": 0.0, "phi": 0.0, "K1": 0.0, "K2": 0.0, "Ms": 0.0, "A": 0.0},
        ]),
        parameters=Parameters(
            size=1.0e-9, scale=0, m_vect=[0, 0, 1], hstart=hs * MU0, hfinal=hf * MU0, hstep=hp * MU0,
            h_vect=[0.01745, 0, 0.99984], mstep=0.4, mfinal=-1.2, tol_fun=1e-10, tol_hmag_factor=1,
            precond_iter=10,
        ),
    )
    sim.run_loop(outdir=outdir, name="hystloop", **loop_kw)
    df = pd.read_csv(f"{outdir}/hystloop.dat", delimiter=" ",
                     names=["configuration_type", "mu0_Hext", "polarisation", "energy_density"])
    return Result(
        H=df["mu0_Hext"].to_numpy() / MU0,
        M=df["polarisation"].to_numpy() / MU0,
        energy_density=df["energy_density"].to_numpy(),
        configurations={i + 1: f for i, f in enumerate(sorted(pathlib.Path(outdir).resolve().glob("*.vtu")))},
        configuration_type=df["configuration_type"].to_numpy(),
    )


def coercivity_remanence(rows):
    """Coercive field and remanence of a descending loop, from ``.dat`` rows
    ``[counter, mu0 Hext, mh, energy]`` (the reference computes neither; ``Result`` holds only
    H and M): ``Hc = |mu0 H|`` where ``mh`` first crosses zero and ``Mr = mh`` at ``H = 0``,
    both by linear interpolation between adjacent field steps, in tesla; NaN when the loop
    does not reach them."""
    rows = np.asarray(rows, dtype=np.float64)
    h, mh = rows[:, 1], rows[:, 2]
    hc = mr = float("nan")
    for i in range(len(h) - 1):
        if mh[i] > 0 >= mh[i + 1] and np.isnan(hc):
            hc = abs(h[i] + (h[i + 1] - h[i]) * mh[i] / (mh[i] - mh[i + 1]))
        if h[i] >= 0 >= h[i + 1] and np.isnan(mr) and h[i] != h[i + 1]:
            mr = mh[i] + (mh[i + 1] - mh[i]) * (0 - h[i]) / (h[i + 1] - h[i])
    return hc, mr


@dataclasses.dataclass(frozen=True)
class Result:
    """Hysteresis loop result."""

    H: np.ndarray
    """External field strengths, A/m."""
    M: np.ndarray
    """Magnetisation along the field for each field strength, A/m."""
    energy_density: np.ndarray | None = None
    """Energy densities, J/m^3."""
    configuration_type: np.ndarray | None = None
    """Index of the representative configuration of each field strength."""
    configurations: dict | None = None
    """Configuration index -> ``.vtu`` path."""

    @property
    def dataframe(self) -> pd.DataFrame:
        return pd.DataFrame({"configuration_type": self.configuration_type, "H": self.H, "M": self.M,
                             "energy_density": self.energy_density})
