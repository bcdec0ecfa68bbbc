"""Benchmark of the hysteresis hot path: field steps per second on the B200 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload large|multigrain|single|batch]

The default workload is the large multigrain cube: 200 nm edge, 80^3 cells x 6 tets
(3,072,000 tets, 531,441 nodes), 27 seeded Voronoi grains with easy axes in a 20 degree cone,
a 2 nm grain-boundary phase (A=2e-12 J/m, K1=0, Js=0.5 T), field along z from +8 T to -8 T in
0.05 T steps (321 field steps, the reference's loop, scripts/loop.py:71-124).  Inputs are
seeded synthetic data of those shapes.

Each path ("variant") first runs the whole sweep once, one field step per launch, untimed:
that gives its coercive field Hc and remanence Mr, its per-step counters and the state
(m, u) before every field step of a window of consecutive field steps around the switching
field (located on the plain FP64 sweep: the steps where the most work is).  A timed "step" is
then one field step of that window, started from its saved state (the state restored before
each step), cycling through the window; ``value`` is field steps per second of the path the
metric names -- mixed precision with the learned warm start, here with the two-level Poisson
preconditioner (``config.path``) -- with the operators resident in HBM (device time from CUDA
events on the library's stream, the L2 flushed before each step).  ``variants`` holds every
path of the same run: the plain FP64 path (the reference's method: the denominator), mixed
precision, mixed with the two-level preconditioner, and the learned start with and without
its residual gate, each with the window rate, the whole-sweep rate, PCG iterations per solve,
Hc/Mr and their deviation from the FP64 path (and from the FP64 oracle's sweep where one is
committed, tests/golden/sweep_*.npz).  ``e2e`` is the headline path through the public API
from pinned host buffers: the mesh built once (a preprocessing-cache hit), then per step the
state uploaded, the field step run and the state read back.  ``cpu_baseline`` is the NumPy
oracle on a bounded sample of the same workload (field step 1 from the initial state), timed
in a separate process on the host cores meanwhile, beside the GPU paths' rates on that same
field step.  Multi-GPU runs are independent replicas (one per rank, no collective on the data
path).  ``--impl reference`` times the CPU oracle alone on the same workload (the reference's
algorithm restated; its own JAX/escript stack is not installable here).
"""

from __future__ import annotations

import argparse
import collections
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
for _p in (ROOT, ROOT / "mammos-mumag_b200"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))

import numpy as np  # noqa: E402

METRIC = "field steps/s + PCG iters/solve: learned+mixed vs plain FP64 GPU at |ΔHc|<1%"
UNIT = "field steps/s"
L2_FLUSH_BYTES = 256 << 20
DBL_MAX = 1.7976931348623157e308
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte of one k_solve
# field-step launch, from one ncu capture (profiles/k_solve_large_mixed_coarse_traffic.md): field
# step 2 of the large mesh on the mixed path with the two-level preconditioner (the headline's
# kernel; its gated learned start ran on none of that step's solves) moved 28.74 GB of DRAM
# traffic for 40.515 GB of algorithmic bytes (the FP32 Poisson operator stays in L2).  The bench
# scales the ratio to its own average launch (traffic grows with the work counters the
# algorithmic bytes are computed from).
TRAFFIC_PER_ALGORITHMIC_BYTE = {("large", "learned_mixed_coarse"): 28.741132032 / 40.515,
                                ("large", "mixed_coarse"): 28.741132032 / 40.515}

# Seeded synthetic workloads: mesh (synthetic.multigrain / single_grain arguments), field
# tilt from z toward x (degrees), sweep (hstart, hfinal, hstep, mstep, mfinal), aggregate
# size of the two-level preconditioner, length of the timed window (field steps), the oracle
# sweep committed for it (tests/golden), description.
WORKLOADS = {
    "large": dict(
        mesh=dict(kind="multigrain", n=80, L=200.0, grains=27, cone_deg=20.0, gb=2.0), tilt=0.0,
        sweep=(8.0, -8.0, -0.05, 0.4, -2.0), coarse=512, window=12, oracle=None, train_seeds=2,
        train_steps=20,
        desc="large multigrain 200 nm, 80^3 x 6 tets (3,072,000 tets, 531,441 nodes), 27 Voronoi grains "
             "(20 deg cone) + 2 nm grain-boundary phase, field along z, +8 -> -8 T in 0.05 T steps "
             "(321 field steps)"),
    "multigrain": dict(
        mesh=dict(kind="multigrain", n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0), tilt=1.0,
        sweep=(8.0, -8.0, -0.1, 0.4, -2.0), coarse=256, window=12, oracle="sweep_multigrain.npz",
        train_seeds=4, train_steps=0,
        desc="multigrain 80 nm, 32^3 x 6 tets (196,608 tets, 35,937 nodes), 8 Voronoi grains "
             "(15 deg cone) + 2 nm grain-boundary phase, field 1 deg off z, +8 -> -8 T in 0.1 T "
             "steps (161 field steps)"),
    "single": dict(
        mesh=dict(kind="single_grain", n=16, L=20.0), tilt=0.0,
        sweep=(8.0, -8.0, -0.2, 0.4, -2.0), coarse=64, window=8, oracle="sweep_single.npz",
        train_seeds=0, train_steps=0,
        desc="single grain 20 nm, 16^3 x 6 tets (24,576 tets, 4,913 nodes), Js=1.61 T, "
             "A=7.7e-12 J/m, K1=4.3e6 J/m^3, +8 -> -8 T in 0.2 T steps (81 field steps)"),
}


def workload(name: str, seed: int = 0):
    """(X, T, tag, krn, m0, hdir) of a workload, from its seed."""
    from mammos_mumag import synthetic

    w = WORKLOADS[name]
    mesh = dict(w["mesh"])
    kind = mesh.pop("kind")
    X, T, tag, krn, m0 = getattr(synthetic, kind)(seed=seed, **mesh)
    d = math.radians(w["tilt"])
    return X, T, tag, krn, m0, [math.sin(d), 0.0, math.cos(d)]


def headline_of(name: str) -> str:
    return "learned_mixed_coarse" if WORKLOADS[name]["train_seeds"] > 0 else "mixed_coarse"


def config_of(name: str, world: int) -> dict:
    """The run's configuration: static, so the reference arm prints the same dictionary."""
    w = WORKLOADS[name]
    head = headline_of(name)
    return {
        "workload": w["desc"],
        "step": (f"one field step of a {w['window']}-step window around the switching field, from its "
                 "saved state (restored before each step)"),
        "path": head,
        "precision": "mixed (FP32 operator planes and inner PCG, FP64 refinement, reductions, energies)",
        "preconditioner": f"two-level additive (Jacobi + {w['coarse']}-node box aggregates); FP64 path: Jacobi",
        "warm_start": "learned (residual-gated)" if head.startswith("learned") else "previous u (reference)",
        "parallelism": f"replicas x{world}",
        "l2": "256 MB buffer written before every timed step (L2 flush)",
    }


def algorithmic_bytes(steps, Z: int, N: int, mixed: bool, coarse: bool) -> float:
    """Compulsory bytes of the persistent field-step kernel, summed over its work counters.

    Z = unpadded node-pair entries, N = nodes; operator values in FP32 (4 B) for the mixed
    path, FP64 (8 B) otherwise; vectors FP64 except the PCG's FP32 inner vectors.
    Per Poisson PCG iteration: the S SpMV Z(s+4) + 4(N+1) + 2Ns and the vector update 9Ns
    (+ Ns for the stored z with the two-level preconditioner).  Per energy evaluation outside
    the PCG: divergence and initial residual Z(3s+8+4) + 5N*8, exchange/anisotropy/gradient
    gathers Z(10s+4) + 14N*8, the normalised trial point 9N*8.  Per M_inv iteration: the C SpMV
    Z(7s+4) + 30N*8.  Per NCG iteration: ~12 three-vector passes 36N*8.  The mixed path's
    refinement passes are not counted (a lower bound).
    """
    s = 4 if mixed else 8
    pcg = sum(st["pcg_iters"] for st in steps)
    ev = sum(st["evals"] for st in steps)
    mi = sum(st["minv_iters"] for st in steps)
    ncg = sum(st["ncg_iters"] for st in steps)
    b = pcg * (Z * (s + 4) + 4 * (N + 1) + 2 * N * s + 9 * N * s + (N * s if coarse else 0))
    b += ev * (Z * (3 * s + 12) + 5 * N * 8 + Z * (10 * s + 4) + 14 * N * 8 + 9 * N * 8)
    b += mi * (Z * (7 * s + 4) + 30 * N * 8)
    b += ncg * 36 * N * 8
    return float(b)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for ln in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in ln.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def batch_workload(count: int = 64, seed: int = 0):
    """64 independent loops on seeded meshes of uneven size: structured grids of 12..40 cells
    per edge (h = 1.25 nm), 6 tets per cell, 1..27 Voronoi grains with easy axes in a cone of
    up to 30 degrees, the single-grain material, a 2 nm grain-boundary phase."""
    from mammos_mumag import synthetic

    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        n = int(rng.integers(12, 41))
        grains = int(rng.integers(1, 28))
        cone = float(rng.uniform(0.0, 30.0))
        out.append(synthetic.multigrain(n=n, L=1.25 * n, grains=grains, cone_deg=cone, gb=2.0 if grains > 1 else 0.0,
                                        seed=seed * 1000 + q))
    return out


_ORACLE = {}


def oracle_step(name: str):
    """One bounded sample of the reference's algorithm on the host: field step 1 of the
    workload's sweep from its initial state (u = 0), by the NumPy/SciPy oracle (the
    reference's scripts/loop.py restated), single-threaded.  The oracle's operators are built
    once per process (untimed).  Returns (seconds, evaluations, PCG iterations)."""
    import oracle as O

    if name not in _ORACLE:
        X, T, tag, krn, m0, hdir = workload(name, 0)
        _ORACLE[name] = (O.Problem(X, T, tag, krn), m0, hdir)
    P, m0, hdir = _ORACLE[name]
    hstart, hfinal, hstep, mstep, mfinal = WORKLOADS[name]["sweep"]
    par = dict(hdir=hdir, hstart=hstart, hfinal=hfinal, hstep=hstep, mstep=mstep, mfinal=mfinal,
               tol_fun=1e-10, tol_u=1e-10, precond_iter=10, hmag_on=1, m=[0.0, 0.0, 1.0])
    t = time.perf_counter()
    _, st = O.run_loop(P, par, m0=m0, max_steps=1)
    return time.perf_counter() - t, st[0].evals, st[0].pcg_iters


def _oracle_job(name):
    return oracle_step(name)


def _cpu_baseline_proc(name, q):
    """cpu_baseline in a separate (spawned) process, alongside the GPU work."""
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    try:
        dt, ev, pcg = oracle_step(name)
        q.put({"seconds": dt, "evals": ev, "pcg_iters": pcg})
    except Exception as e:  # reported, not fatal
        q.put({"error": repr(e)})


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def host_memory_available():
    """Bytes of host memory this process may still use: the host's available memory, capped
    by the memory cgroup's limit less its usage (v2 or v1 files) where one is set; None if
    unknown."""
    avail = None
    try:
        import psutil

        avail = psutil.virtual_memory().available
    except Exception:
        pass
    for lim, use in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            text = pathlib.Path(lim).read_text().strip()
            if text == "max" or int(text) >= 1 << 60:
                break
            left = max(0, int(text) - int(pathlib.Path(use).read_text().strip()))
            avail = left if avail is None else min(avail, left)
            break
        except (OSError, ValueError):
            continue
    return avail


def _reference_samples(workload, procs, warm, steps):
    """``warm`` untimed then ``steps`` timed oracle samples in ``procs`` spawned processes
    (each process builds the oracle's operators on its first sample, untimed).  Returns the
    samples and the wall time of the timed ones."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    with ProcessPoolExecutor(max_workers=procs, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_oracle_job, [workload] * warm))
        t0 = time.perf_counter()
        res = list(ex.map(_oracle_job, [workload] * steps))
        return res, time.perf_counter() - t0


def run_reference(args, world, rank):
    """The reference's algorithm on the host cores: the oracle port (the reference's own
    esys-escript/JAX stack is not installable here), on the same workload and configuration
    as the GPU arm.  A step is one bounded sample of that workload -- field step 1 of its
    sweep from the initial state, single-threaded (one sweep is sequential and the port's
    sparse kernels are single-threaded).  The samples run in P spawned processes at once so
    the run ends within minutes on the large mesh, whose field step takes tens of seconds
    here; value = 1 / mean sample time, the rate of one sweep (the concurrent samples share
    memory bandwidth, so it is if anything low).  Under torchrun rank 0 alone runs."""
    if rank != 0:
        return 0
    from concurrent.futures.process import BrokenProcessPool

    cores = host_cores()
    avail = host_memory_available()
    # peak resident memory of one sample process (the oracle's operator build): 7.3 GB
    # measured on the large mesh, ~15x less on the multigrain one
    per_proc = {"large": 9 << 30, "multigrain": 1 << 30, "single": 1 << 29}[args.workload]
    procs = max(1, min(8, cores, args.steps + args.warmup,
                       int(avail // per_proc) if avail else 8))
    if args.ref_procs > 0:
        procs = min(procs, args.ref_procs)
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    # A sample process that dies (the kernel's out-of-memory killer) breaks the executor with
    # an error instead of leaving the map waiting: retry with half the processes, down to one.
    while True:
        try:
            res, wall = _reference_samples(args.workload, procs, max(args.warmup, procs), args.steps)
            break
        except BrokenProcessPool as e:
            if procs == 1:
                print(json.dumps({"impl": "reference", "unavailable": f"the oracle's sample process died ({e!r}); "
                                  f"it needs about {per_proc >> 30} GB of host memory"}), flush=True)
                return 0
            procs = max(1, procs // 2)
    secs = [r[0] for r in res]
    v = len(secs) / sum(secs)
    sample = (f"field step 1 of the sweep from the initial state (u = 0) per step, NumPy/SciPy oracle, "
              f"single-threaded, {procs} samples at a time in separate processes; value = 1 / mean sample "
              f"time ({statistics.mean(secs):.1f} s; {res[0][1]} energy evaluations, {res[0][2]} PCG iterations)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args.workload, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "host_cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_sweep(M, m0, sweep, sp, window=0, keep=None):
    """The reference's field loop (scripts/loop.py:71-124: cumulative field, mfinal stop,
    snapshot counter) one field step per launch, untimed.  Keeps the state (m, u, field)
    before the steps in ``keep``; with ``keep`` None it locates the switching step (the
    first whose mh is <= 0) and keeps the ``window`` steps around it.  Returns (rows, step
    dicts, kept states, first window step)."""
    hstart, hfinal, hstep, mstep, mfinal = sweep
    nmax = int(abs(hfinal - hstart) / abs(hstep)) + 1
    M.set_state(m0, None, m0)
    rows, steps, states = [], [], {}
    recent = collections.deque(maxlen=window // 2 + 1) if keep is None else None
    want = set(keep) if keep is not None else set()
    j0 = None
    mh = last = DBL_MAX
    counter, h = 0, hstart
    for idx in range(nmax):
        if not mh > mfinal:
            break
        if recent is not None or idx in want:
            m, u, _ = M.get_state()
            if idx in want:
                states[idx] = (m, u, h)
            if recent is not None:
                recent.append((idx, m, u, h))
        r = M.minimize(h, sp)
        if r["status"] != 0:
            raise RuntimeError(f"field step {idx} returned status {r['status']}")
        mh = r["mh"]
        if (last - mh) > mstep:
            counter += 1
            last = mh
        rows.append([counter, h, mh, r["energy"]])
        steps.append(r)
        if recent is not None and mh <= 0.0:  # switching: the window is half before, half after
            j0 = max(0, idx - window // 2)
            for j, m, u, hj in recent:
                if j >= j0:
                    states[j] = (m, u, hj)
            want = set(range(idx + 1, j0 + window))
            recent = None
        h = h + hstep
    rows = np.array(rows)
    if keep is None and j0 is None:  # no switching within the sweep: the last steps
        raise RuntimeError("the sweep does not switch; no window to time")
    return rows, steps, states, j0


def time_window(M, states, order, sp, m0, flush, warmup, steps, world):
    """W untimed, then K timed field steps cycling through ``order``, each from its saved
    state, the L2 flushed before each, device time from CUDA events on the library's stream.
    Returns (ms over ranks, step dicts)."""
    import torch

    def one(t, timed):
        m, u, h = states[order[t % len(order)]]
        M.set_state(m, u, m0)
        if timed:
            flush.fill_(1.0)  # L2 flush (256 MB > 126 MB L2)
            torch.cuda.synchronize()
            M.timer_start()
        r = M.minimize(h, sp)
        return (M.timer_stop() if timed else 0.0), r

    for t in range(warmup):
        one(t, False)
    dist_barrier(world)
    torch.cuda.synchronize()
    total, out = 0.0, []
    for t in range(steps):
        ms, r = one(t, True)
        total += ms
        out.append(r)
    torch.cuda.synchronize()
    dist_barrier(world)
    return dist_max(total, world), out


def train_model(name, rank, local):
    """The learned start's network, trained at set-up (untimed) on plain loops of other seeds
    of the workload's mesh family."""
    from mammos_mumag import learned

    w = WORKLOADS[name]
    mesh = w["mesh"]
    hs = w["sweep"]
    spec = learned.LoopSpec(n=mesh["n"], L=mesh["L"], grains=mesh["grains"], cone_deg=mesh["cone_deg"],
                            gb=mesh["gb"], hstart=hs[0], hfinal=hs[1], hstep=hs[2], tilt_deg=w["tilt"],
                            max_steps=w["train_steps"])
    t0 = time.perf_counter()
    feats, targets = learned.collect([1000 + 10 * rank + q for q in range(w["train_seeds"])], spec,
                                     samples=50000, device=local)
    t1 = time.perf_counter()
    model, loss = learned.train(feats, targets, epochs=30, device=local)
    info = {"samples": int(len(targets)), "training_meshes": w["train_seeds"], "collect_s": t1 - t0,
            "train_s": time.perf_counter() - t1, "loss_rel": loss}
    return model, info


def variant_table(name, gate):
    """(variant, precision, aggregate nodes, learned gate or None); the first is the plain
    FP64 path (the reference's method, the denominator)."""
    from mammos_mumag import _native

    cb = WORKLOADS[name]["coarse"]
    out = [("fp64", _native.PREC_FP64, 0, None), ("mixed", _native.PREC_MIXED, 0, None),
           ("mixed_coarse", _native.PREC_MIXED, cb, None)]
    if WORKLOADS[name]["train_seeds"] > 0:
        out.append(("learned_mixed_coarse", _native.PREC_MIXED, cb, gate))
    return out


def hc_mr(rows):
    from mammos_mumag.hysteresis import coercivity_remanence

    return coercivity_remanence(rows)


def rel(a, b):
    return abs(a - b) / abs(b) if np.isfinite(a) and np.isfinite(b) and b != 0 else None


def run_b200(args, world, rank, local):
    import multiprocessing as mp

    import torch

    from mammos_mumag import _native

    if _native.device_count() < 1:
        raise RuntimeError("no sm_100 GPU visible")
    torch.cuda.set_device(local)
    name = args.workload
    w = WORKLOADS[name]
    X, T, tag, krn, m0, hdir = workload(name, 0)
    sp = _native.solver_params(hdir=hdir)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    head = headline_of(name)
    # the CPU oracle's sample, in its own process while the GPU works (rank 0, one GPU)
    cpu_q = cpu_p = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ctx = mp.get_context("spawn")
        cpu_q = ctx.Queue()
        cpu_p = ctx.Process(target=_cpu_baseline_proc, args=(name, cpu_q), daemon=True)
        cpu_p.start()
    model, train_info = (None, None)
    if w["train_seeds"] > 0:
        model, train_info = train_model(name, rank, local)

    def make_mesh(prec, cb, gate):
        msh = _native.Mesh(X, T, tag, krn, device=local, precision=prec, coarse_box_nodes=cb)
        if gate is not None:
            msh.set_warm_start(_native.WARM_LEARNED, model)
            msh.set_learned_gate(gate)
        msh.set_state(m0, None, m0)
        msh.autotune(sp)  # launch shape (set-up, untimed)
        return msh

    variants, runs = {}, {}
    j0, order = None, None
    for vname, prec, cb, gate in variant_table(name, args.learned_gate):
        msh = make_mesh(prec, cb, gate)
        info = msh.info()
        keep = None if j0 is None else order
        rows, steps, states, jw = run_sweep(msh, m0, w["sweep"], sp, window=w["window"], keep=keep)
        if j0 is None:  # the plain FP64 sweep locates the window
            j0 = jw
            order = [j for j in range(j0, j0 + w["window"]) if j in states]
        clk = ClockSampler(local) if vname == head else None
        if clk:
            clk.__enter__()
        try:
            ms, tsteps = time_window(msh, states, order, sp, m0, flush, args.warmup, args.steps, world)
        finally:
            if clk:
                clk.__exit__(None, None, None)
        # the restored steps repeat the sweep's own steps (deterministic kernels: identical energies)
        restored = max(abs(r["energy"] - rows[order[t % len(order)]][3]) / abs(rows[order[t % len(order)]][3])
                       for t, r in enumerate(tsteps))
        hc, mr = hc_mr(rows)
        ev = sum(s["evals"] for s in tsteps)
        sev = sum(s["evals"] for s in steps)
        variants[vname] = {
            "value": len(tsteps) * world / (ms * 1e-3),
            "pcg_iters_per_solve": sum(s["pcg_iters"] for s in tsteps) / max(1, ev),
            "sweep_value": len(steps) / (1e-3 * sum(s["device_ms"] for s in steps)),
            "sweep_pcg_iters_per_solve": sum(s["pcg_iters"] for s in steps) / max(1, sev),
            "sweep_steps": len(steps),
            "hc_T": hc, "mr_T": mr,
            "learned_starts_per_solve": (sum(s["learned_starts"] for s in steps) / max(1, sev)
                                         if gate is not None else None),
            "learned_gate": gate,
            "grid_ctas": info["grid_ctas"], "kernel_ctas_per_sm": info["kernel_ctas_per_sm"],
            "pcg_variant": info["pcg_variant"], "coarse_boxes": info["coarse_boxes"],
            "restored_energy_dev": restored,
        }
        runs[vname] = dict(ms=ms, tsteps=tsteps, steps=steps, rows=rows, info=info, clk=clk, states=states,
                           prec=prec, cb=cb, gate=gate)
        if vname == head and gate is not None:
            # the same window with the learned start on every solve (no gate), on this path's states
            msh.set_learned_gate(0.0)
            ms_u, ts_u = time_window(msh, states, order, sp, m0, flush, args.warmup, args.steps, world)
            evu = sum(s["evals"] for s in ts_u)
            variants[vname + "_ungated"] = {
                "value": len(ts_u) * world / (ms_u * 1e-3),
                "pcg_iters_per_solve": sum(s["pcg_iters"] for s in ts_u) / max(1, evu),
                "learned_starts_per_solve": sum(s["learned_starts"] for s in ts_u) / max(1, evu),
                "note": "window only, from the gated path's saved states",
            }
        msh.close()
    return finish_b200(args, world, rank, local, name, variants, runs, head, j0, order, model, train_info,
                       cpu_q, cpu_p, sp, m0, X, T, tag, krn, flush)


def run_batch(args, world, rank, local):
    """The batched workload: 64 independent loops on seeded meshes of uneven size, the whole
    sweep of all 64 meshes in ONE persistent launch (mm_batch_loop: a CTA group per mesh
    runs that mesh's field steps on the device).  Beside it, the same loops run one after
    another with their own autotuned launches (one launch per field step)."""
    import torch

    from mammos_mumag import _native

    torch.cuda.set_device(local)
    data = batch_workload(64, seed=rank)
    sp = _native.solver_params(hdir=[0.0, 0.0, 1.0])
    sw = (8.0, -8.0, -0.2, 0.4, -2.0)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    variants, clk = {}, None
    for name, prec in (("fp64", _native.PREC_FP64), ("mixed", _native.PREC_MIXED)):
        meshes = [_native.Mesh(X, T, tag, krn, device=local, precision=prec) for X, T, tag, krn, _ in data]
        try:
            def reset():
                for M, d in zip(meshes, data):
                    M.set_state(d[4], None, d[4])

            with _native.Batch(meshes) as B:
                for _ in range(args.warmup):
                    reset()
                    B.loop(*sw, sp)
                t_ms, nfs, pcg, ev = 0.0, 0, 0, 0
                dist_barrier(world)
                with ClockSampler(local) as c:
                    for _ in range(args.steps):
                        flush.fill_(1.0)
                        torch.cuda.synchronize()
                        reset()
                        B.timer_start()
                        out = B.loop(*sw, sp)
                        t_ms += B.timer_stop()
                        for rows, st in out:
                            nfs += len(rows)
                            pcg += sum(x["pcg_iters"] for x in st)
                            ev += sum(x["evals"] for x in st)
                if name == "fp64":
                    clk = c
                groups = B.groups()
            t_ms = dist_max(t_ms, world)
            variants[name] = {"value": nfs * world / (t_ms * 1e-3), "pcg_iters_per_solve": pcg / max(1, ev),
                              "ms_per_sweep": t_ms / args.steps, "ctas": int(groups[-1])}
            # the same loops one after another, each with its own autotuned launch shape
            seq_ms, seq_n = 0.0, 0
            for M, d in zip(meshes, data):
                M.set_state(d[4], None, d[4])
                M.autotune(sp)
                M.set_state(d[4], None, d[4])
                M.loop(*sw, sp)  # warm-up
                M.set_state(d[4], None, d[4])
                M.timer_start()
                rows, _ = M.loop(*sw, sp)
                seq_ms += M.timer_stop()
                seq_n += len(rows)
            seq_ms = dist_max(seq_ms, world)
            variants[name + "_sequential"] = {"value": seq_n * world / (seq_ms * 1e-3), "ms_per_sweep": seq_ms}
        finally:
            for M in meshes:
                M.close()
    if rank == 0:
        nodes = [d[0].shape[0] for d in data]
        line = {
            "metric": "field steps/s (sum over the batch's loops)", "value": variants["fp64"]["value"],
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": variants["fp64"]["ms_per_sweep"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": ("64 independent loops, seeded structured meshes of 12..40 cells per edge "
                                    f"(h = 1.25 nm, {min(nodes)}..{max(nodes)} nodes), 1..27 Voronoi grains, cone "
                                    "<= 30 deg, +8 -> -8 T in 0.2 T steps (81), all sweeps in one persistent "
                                    "launch"),
                       "parallelism": f"replicas x{world}", "l2": "256 MB buffer written between timed sweeps"},
            "variants": variants,
            "gpu_launches": args.steps,
            "clocks": clk.summary() if clk is not None else None,
        }
        print(json.dumps(line), flush=True)
    return 0


def finish_b200(args, world, rank, local, name, variants, runs, head, j0, order, model, train_info, cpu_q, cpu_p,
                sp, m0, X, T, tag, krn, flush):
    import torch

    from mammos_mumag import _native

    w = WORKLOADS[name]
    ref = variants["fp64"]
    oracle_hc = oracle_mr = None
    if w["oracle"]:
        f = np.load(ROOT / "tests" / "golden" / w["oracle"])
        oracle_hc, oracle_mr = float(f["hc"]), float(f["mr"])
    for vname, v in variants.items():
        if vname != "fp64":
            v["speedup_vs_fp64"] = v["value"] / ref["value"]
            v["pcg_per_solve_vs_fp64"] = v["pcg_iters_per_solve"] / ref["pcg_iters_per_solve"]
        if "hc_T" not in v:
            continue
        if vname != "fp64":
            v["sweep_speedup_vs_fp64"] = v["sweep_value"] / ref["sweep_value"]
            v["dHc_rel"] = rel(v["hc_T"], ref["hc_T"])
            v["dMr_rel"] = rel(v["mr_T"], ref["mr_T"])
        if oracle_hc is not None:
            v["dHc_rel_oracle"] = rel(v["hc_T"], oracle_hc)
            v["dMr_rel_oracle"] = rel(v["mr_T"], oracle_mr)
    hr = runs[head]
    value = variants[head]["value"]
    tsteps = hr["tsteps"]
    launches = len(tsteps)
    kernel_ms = sum(s["device_ms"] for s in tsteps)
    Z, N = hr["info"]["nnz"], hr["info"]["nodes"]
    ab = algorithmic_bytes(tsteps, Z, N, mixed=hr["prec"] == _native.PREC_MIXED, coarse=hr["cb"] > 0)
    achieved = ab / (kernel_ms * 1e-3) / 1e9  # GB/s over the kernel's own launch durations
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    ratio = TRAFFIC_PER_ALGORITHMIC_BYTE.get((name, head))
    traffic = ratio * ab / launches if ratio is not None else None
    # e2e: the public API from pinned host buffers -- the mesh built once (the preprocessing
    # cache hits: X, T, tag are hashed and compared), then per step the state uploaded, the
    # field step run and the state read back
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    pX, pT, ptag, pm0 = pin(X), pin(np.asarray(T, np.int32)), pin(np.asarray(tag, np.int32)), pin(m0)
    pstates = {j: (pin(m), pin(u), h) for j, (m, u, h) in hr["states"].items()}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with _native.Mesh(pX, pT, ptag, krn, device=local, precision=hr["prec"], coarse_box_nodes=hr["cb"]) as mm:
        if hr["gate"] is not None:
            mm.set_warm_start(_native.WARM_LEARNED, model)
            mm.set_learned_gate(hr["gate"])
        mm.set_state(pm0, None, pm0)
        mm.autotune(sp)  # cached for this mesh shape: no timing runs
        for t in range(args.steps):
            m, u, h = pstates[order[t % len(order)]]
            mm.set_state(m, u, pm0)
            mm.minimize(h, sp)
            mout, uout, gout = mm.get_state()
    e2e_t = time.perf_counter() - t0
    e2e_t = dist_max(e2e_t, world)
    h2d = 8 * (3 * N + N + 3 * N) + (pX.nbytes + pT.nbytes + ptag.nbytes + 48 * len(krn)) / args.steps
    d2h = 8 * (3 * N + N + 3 * N) + 128
    if rank != 0:
        return 0
    cpu = None
    if cpu_p is not None:
        cpu_p.join(timeout=1800)
        res = (cpu_q.get(timeout=5) if not cpu_q.empty()
               else {"error": f"no result (sample process exit code {cpu_p.exitcode}; -9: killed, e.g. out of memory)"})
        if "seconds" in res:
            same = {k: 1e3 / runs[k]["steps"][0]["device_ms"] for k in ("fp64", head)}
            cpu = {"value": 1.0 / res["seconds"], "unit": UNIT, "cores": 1, "host_cores": host_cores(), "kind": "port",
                   "sample": (f"field step 1 of the sweep from the initial state (u = 0), NumPy/SciPy oracle, "
                              f"single thread, {res['seconds']:.1f} s ({res['evals']} energy evaluations, "
                              f"{res['pcg_iters']} PCG iterations), run in a separate process during the GPU work"),
                   "gpu_same_sample": {k: {"value": v, "ratio_to_cpu": v * res["seconds"]} for k, v in same.items()}}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "port", "error": res.get("error")}
    clk = hr["clk"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": hr["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": config_of(name, world),
        "window": {"first_step": j0, "steps": len(order),
                   "fields_T": [hr["states"][order[0]][2], hr["states"][order[-1]][2]],
                   "located_by": "the plain FP64 sweep's first field step with mh <= 0, half the window before it"},
        "pcg_iters_per_solve": variants[head]["pcg_iters_per_solve"],
        "speedup_vs_fp64": variants[head]["speedup_vs_fp64"],
        "hc_T": variants[head]["hc_T"], "mr_T": variants[head]["mr_T"],
        "dHc_rel": variants[head].get("dHc_rel"), "dMr_rel": variants[head].get("dMr_rel"),
        "variants": variants,
        "learned_training": train_info,
        "launch": {"grid_ctas": hr["info"]["grid_ctas"], "block_threads": hr["info"]["block_threads"],
                   "kernel_ctas_per_sm": hr["info"]["kernel_ctas_per_sm"]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "traffic_source": ("DRAM bytes per algorithmic byte of one ncu-captured field-step launch of "
                                        "this path, scaled to the average launch") if traffic is not None else None,
                     "kernel": f"k_solve (persistent field step, {head})",
                     "algorithmic_bytes_per_launch": ab / launches, "avg_launch_ms": kernel_ms / launches,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
        "cpu_baseline": cpu,
        "e2e": {"value": args.steps * world / e2e_t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h),
                "includes": "mesh build (preprocessing-cache hit) once, then per step state upload, field step, "
                            "state read-back"},
        "gpu_launches": launches,
        "clocks": clk.summary() if clk is not None else None,
    }
    print(json.dumps(line), flush=True)
    if model is not None:
        model.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["large", "multigrain", "single", "batch"], default="large")
    ap.add_argument("--learned-gate", type=float, default=1e8,
                    help="the learned start runs only on solves whose initial residual exceeds this many "
                         "times the stop tolerance (0: every solve)")
    ap.add_argument("--ref-procs", type=int, default=0,
                    help="reference arm: at most this many concurrent sample processes (0: up to 8)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            if args.workload == "batch":
                raise SystemExit("the reference arm times the single-sweep workloads")
            return run_reference(args, world, rank)
        if args.workload == "batch":
            return run_batch(args, world, rank, local)
        return run_b200(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
