"""Regenerate the oracle's full field sweeps of the single-grain and multigrain workloads.

The reference records no loop that crosses the coercive field (its only loop golden,
``tests/data/loop/cube.dat``, stops at +0.2 T), and its bare-box boundary branch, which every
synthetic workload takes, has no golden at all.  These fixtures are therefore the FP64 oracle's
own sweeps (``oracle/mumag_oracle.py``, itself pinned to the reference's goldens) through
switching, so the GPU path's rows, coercivity and remanence can be compared with it:

* ``sweep_single.npz``     -- one cubic grain, 20 nm, 16^3 x 6 tets (4,913 nodes), Js=1.61 T,
                              A=7.7e-12 J/m, K1=4.3e6 J/m^3, easy axis +z, m0 = +z plus a seeded
                              Gaussian perturbation (sigma 0.01, seed 0), field along +z from
                              +8 T to -8 T in 0.2 T steps, mfinal = -2 (all 81 steps);
* ``sweep_multigrain.npz`` -- 80 nm cube, 32^3 x 6 tets (35,937 nodes), 8 Voronoi grains
                              (15 degree cone, seed 0) + 2 nm grain-boundary phase, field 1
                              degree off z toward x, +8 T to -8 T in 0.1 T steps (161 steps).

Each file holds ``rows`` [n,4] (counter, mu0 Hext, mh, energy in internal units), ``stats``
[n,5] (NCG iterations, evaluations, PCG iterations, line-search halvings, M_inv
iterations), ``hc``/``mr`` (tesla) and the run's parameters.  The meshes are rebuilt from
their seeds by ``mammos_mumag.synthetic`` (the same calls as here).

Usage::

    python tests/golden/make_sweeps.py [single|multigrain ...]
"""

import json
import math
import multiprocessing as mp
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for _p in (ROOT, ROOT / "mammos-mumag_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

CASES = {
    "single": dict(mesh=dict(kind="single_grain", n=16, L=20.0, seed=0), hdir=[0.0, 0.0, 1.0],
                   hstart=8.0, hfinal=-8.0, hstep=-0.2, mstep=0.4, mfinal=-2.0),
    "multigrain": dict(mesh=dict(kind="multigrain", n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0, seed=0),
                       hdir=[math.sin(math.radians(1.0)), 0.0, math.cos(math.radians(1.0))],
                       hstart=8.0, hfinal=-8.0, hstep=-0.1, mstep=0.4, mfinal=-2.0),
}


def build_case(name):
    """(X, T, tag, krn, m0, par) of a case, from its seeds."""
    from mammos_mumag import synthetic

    c = CASES[name]
    mesh = dict(c["mesh"])
    kind = mesh.pop("kind")
    X, T, tag, krn, m0 = getattr(synthetic, kind)(**mesh)
    par = dict(hdir=c["hdir"], hstart=c["hstart"], hfinal=c["hfinal"], hstep=c["hstep"], mstep=c["mstep"],
               mfinal=c["mfinal"], tol_fun=1e-10, tol_u=1e-10, precond_iter=10, hmag_on=1, m=[0.0, 0.0, 1.0])
    return X, T, tag, krn, m0, par


def run_case(name):
    import oracle as O
    from mammos_mumag.hysteresis import coercivity_remanence

    X, T, tag, krn, m0, par = build_case(name)
    P = O.Problem(X, T, tag, krn)
    t0 = time.perf_counter()
    rows, stats = O.run_loop(P, par, m0=m0)
    dt = time.perf_counter() - t0
    st = np.array([[s.ncg_iters, s.evals, s.pcg_iters, s.ls_shrinks, s.minv_iters] for s in stats], np.int64)
    hc, mr = coercivity_remanence(rows)
    np.savez_compressed(HERE / f"sweep_{name}.npz", rows=rows, stats=st, hc=hc, mr=mr,
                        params=json.dumps(CASES[name]))
    return name, len(rows), hc, mr, dt


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    with mp.get_context("spawn").Pool(len(names)) as pool:
        for name, n, hc, mr, dt in pool.map(run_case, names):
            print(f"{name}: {n} rows, Hc {hc:.6f} T, Mr {mr:.6f} T, {dt:.0f} s")
