"""Finite-element micromagnetic simulations (hysteresis) on B200 GPUs.

A drop-in for the hysteresis-loop path of ``mammos_mumag``: the same modules and file
formats, with the loop computed by ``libmumag_b200.so`` (sm_100a CUDA) in process.
"""

import pathlib

from mammos_mumag import fly, hysteresis, materials, mesh, parameters, runner, simulation, synthetic, vtu

__all__ = ["hysteresis", "materials", "mesh", "parameters", "simulation", "fly", "vtu", "synthetic", "runner"]

__version__ = "0.7.1+b200.0.1"
_lib_path = pathlib.Path(__file__).resolve().parent / "lib" / "libmumag_b200.so"
