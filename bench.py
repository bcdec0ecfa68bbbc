"""Benchmark of the hysteresis hot path: field steps per second on the B200 path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload multigrain|single|large|batch]

A step is one full field sweep of the workload (the reference's loop, scripts/loop.py:71-142,
run to the last field value).  The default workload is the multigrain cube: 80 nm edge,
32^3 cells x 6 tets (196,608 tets, 35,937 nodes), 8 seeded Voronoi grains with easy axes in
a 15 degree cone, a 2 nm grain-boundary phase (A=2e-12 J/m, K1=0, Js=0.5 T), field along z
tilted 1 degree toward x, +8 T -> -8 T in 0.1 T steps (161 field steps), FP64.  Inputs are
seeded synthetic data of those shapes.

``value`` is whole-job field steps/s of the path the metric names -- mixed precision with
the learned warm start (``config.path`` = learned_mixed; the plain FP64 path for the
single-grain workload or with ``--no-learned``) -- with the mesh operators resident in HBM
(device time from CUDA events on the library's stream); ``variants`` holds the plain FP64,
mixed and learned+mixed sweeps of the same run with their PCG iterations per solve and
Hc/Mr against FP64.  ``e2e`` is the headline path through the public API from host buffers
(mesh build + state upload + sweep + result read-back), ``cpu_baseline`` the CPU oracle on
a bounded sample.  The network of the learned warm start is trained at set-up (untimed) on
plain loops of other seeds of the same mesh family.  Multi-GPU runs are independent replicas (one sweep per rank,
no collective on the data path).  ``--impl reference`` times the CPU oracle alone (the
reference's algorithm restated; its own JAX/escript stack is not installable here).
"""

from __future__ import annotations

import argparse
import json
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
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte of one
# k_solve field-step launch, from one ncu capture of each workload and path
# (python -m mammos_mumag.perfcase field-step ...): the multigrain FP64 launch moved
# 133.8 MB for 5,422 MB of algorithmic bytes, the multigrain learned+mixed launch (network
# on tcgen05) 406.5 MB for 4,128 MB, the large mesh's FP64 launch 178.3 GB for 162.8 GB.
# The bench scales the ratio to its own average launch (traffic grows with the work
# counters the algorithmic bytes are computed from).
TRAFFIC_PER_ALGORITHMIC_BYTE = {("multigrain", "fp64"): 133.8 / 5422.4,
                                ("multigrain", "learned_mixed"): 406.5 / 4128.4,
                                ("large", "fp64"): 178.3 / 162.8}


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


def workload(name: str, seed: int):
    from mammos_mumag import synthetic

    if name == "large":
        X, T, tag, krn, m0 = synthetic.multigrain(n=80, L=200.0, grains=27, cone_deg=20.0, gb=2.0, seed=seed)
        hdir = [0.0, 0.0, 1.0]
        sweep = dict(hstart=8.0, hfinal=-8.0, hstep=-0.05, mstep=0.4, mfinal=-2.0, max_steps=20)
        desc = ("large multigrain 200 nm, 80^3 x 6 tets (3,072,000 tets, 531,441 nodes), 27 Voronoi grains "
                "(20 deg cone) + 2 nm grain-boundary phase, +8 T in 0.05 T steps, first 20 field steps of 321")
        return X, T, tag, krn, m0, hdir, sweep, desc
    if name == "single":
        X, T, tag, krn, m0 = synthetic.single_grain(16, 20.0, seed=seed)
        hdir = [0.0, 0.0, 1.0]
        sweep = dict(hstart=8.0, hfinal=-8.0, hstep=-0.2, mstep=0.4, mfinal=-2.0)
        desc = ("single grain 20 nm, 16^3 x 6 tets (24,576 tets, 4,913 nodes), Js=1.61 T, "
                "A=7.7e-12 J/m, K1=4.3e6 J/m^3, +8 -> -8 T in 0.2 T steps (81 field steps)")
    else:
        X, T, tag, krn, m0 = synthetic.multigrain(n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0, seed=seed)
        d = np.radians(1.0)
        hdir = [float(np.sin(d)), 0.0, float(np.cos(d))]
        sweep = dict(hstart=8.0, hfinal=-8.0, hstep=-0.1, mstep=0.4, mfinal=-2.0)
        desc = ("multigrain 80 nm, 32^3 x 6 tets (196,608 tets, 35,937 nodes), 8 Voronoi grains "
                "(15 deg cone) + 2 nm grain-boundary phase, field 1 deg off z, +8 -> -8 T in 0.1 T "
                "steps (161 field steps)")
    return X, T, tag, krn, m0, hdir, sweep, desc


def hc_mr(rows):
    """Coercive field and remanence of the sweep's rows (``mammos_mumag.hysteresis``)."""
    from mammos_mumag.hysteresis import coercivity_remanence

    return coercivity_remanence(rows)


def algorithmic_bytes(steps, Z: int, N: int, s: int = 8, s_pcg: int | None = None) -> float:
    """Compulsory bytes of the persistent field-step kernel, summed over its work counters.

    Z = unpadded node-pair entries of the SELL pattern, N = nodes, s = value bytes of the
    energy / NCG / M_inv work, s_pcg = value bytes of the Poisson PCG iterations (4 when they
    run on FP32 planes, mixed precision; default s).
    Per Poisson PCG iteration: one S SpMV Z(s+4) + 4(N+1) + 2Ns and the fused vector
    update 9Ns.  Per energy evaluation outside the PCG: divergence + initial residual
    Z(4s+4) + 5Ns, exchange/anisotropy/gradient gathers Z(10s+4) + 14Ns, the normalised
    trial point 9Ns.  Per M_inv iteration: the C SpMV Z(7s+4) + 6Ns and ~8 three-vector
    passes 24Ns.  Per NCG iteration: ~12 three-vector passes 36Ns.
    """
    sp = s if s_pcg is None else s_pcg
    pcg = sum(st["pcg_iters"] for st in steps)
    ev = sum(st["evals"] for st in steps)
    mi = sum(st["minv_iters"] for st in steps)
    ncg = sum(st["ncg_iters"] for st in steps)
    b = pcg * (Z * (sp + 4) + 4 * (N + 1) + 2 * N * sp + 9 * N * sp)
    b += ev * (Z * (4 * s + 4) + 5 * N * s + Z * (10 * s + 4) + 14 * N * s + 9 * N * s)
    b += mi * (Z * (7 * s + 4) + 30 * N * s)
    b += ncg * 36 * N * s
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


def cpu_sample(name: str, n_field_steps: int, seed: int = 0):
    """The CPU oracle (NumPy/SciPy restatement of the reference's loop) on the first
    ``n_field_steps`` field steps of the workload.  Returns (field steps/s, seconds, threads)."""
    import oracle as O

    X, T, tag, krn, m0, hdir, sweep, _ = workload(name, seed)
    P = O.Problem(X, T, tag, krn)
    par = dict(hdir=hdir, tol_fun=1e-10, tol_u=1e-10, precond_iter=10, hmag_on=1, m=[0, 0, 1.0], **sweep)
    par.pop("max_steps", None)
    t = time.perf_counter()
    rows, _ = O.run_loop(P, par, m0=m0, max_steps=n_field_steps)
    dt = time.perf_counter() - t
    return len(rows) / dt, dt, len(rows)


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


_REF_CACHE = {}


def _ref_sample(job):
    """One bounded sample of the CPU reference path in a worker process: the first
    ``n_fs`` field steps of the workload's sweep.  The oracle's operators are built once
    per process (cached), so repeated samples time the loop alone."""
    import oracle as O

    name, n_fs = job
    if name not in _REF_CACHE:
        X, T, tag, krn, m0, hdir, sweep, _ = workload(name, 0)
        par = dict(hdir=hdir, tol_fun=1e-10, tol_u=1e-10, precond_iter=10, hmag_on=1, m=[0, 0, 1.0], **sweep)
        par.pop("max_steps", None)
        _REF_CACHE[name] = (O.Problem(X, T, tag, krn), par, m0)
    P, par, m0 = _REF_CACHE[name]
    t = time.perf_counter()
    rows, _ = O.run_loop(P, par, m0=m0, max_steps=n_fs)
    return len(rows), time.perf_counter() - t


def run_reference(args, world, rank):
    """The reference's algorithm on the host cores: the oracle port (the reference's own
    esys-escript/JAX stack is not installable here), every step a bounded sample of the
    workload.  One sweep is sequential and the port's sparse kernels (scipy.sparse) are
    single-threaded, so the configured workload -- one sweep -- uses one host core
    (``--ref-procs 1``, the default); ``--ref-procs N`` (0 = one per usable core) runs N
    independent replicas of the sample in parallel processes and reports their summed
    throughput instead."""
    if rank != 0:
        return 0
    import multiprocessing as mp

    n_fs = 4
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    procs = max(1, cores if args.ref_procs <= 0 else min(cores, args.ref_procs))
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"
    jobs = [(args.workload, n_fs)] * procs
    with mp.get_context("spawn").Pool(procs) as pool:
        for _ in range(max(1, args.warmup)):
            pool.map(_ref_sample, jobs, chunksize=1)
        tot_t, tot_n = 0.0, 0
        for _ in range(args.steps):
            t0 = time.perf_counter()
            res = pool.map(_ref_sample, jobs, chunksize=1)
            tot_t += time.perf_counter() - t0
            tot_n += sum(n for n, _ in res)
    v = tot_n / tot_t
    _, _, _, _, _, _, _, desc = workload(args.workload, 0)
    sample = (f"first {n_fs} field steps of the sweep, NumPy/SciPy oracle, single thread" if procs == 1 else
              f"first {n_fs} field steps of the sweep per replica, {procs} single-threaded NumPy/SciPy oracle "
              f"replicas in parallel per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc + f"; each step = the first {n_fs} field steps"
                   + (f", {procs} replicas" if procs > 1 else ""),
                   "precision": "fp64"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def loop_spec(name: str):
    """The workload's mesh family and sweep as a ``learned.LoopSpec`` (training loops for the
    learned warm start run on other seeds of the same family)."""
    from mammos_mumag import learned

    if name == "large":
        return learned.LoopSpec(n=80, L=200.0, grains=27, cone_deg=20.0, gb=2.0, hstep=-0.05, tilt_deg=0.0,
                                max_steps=20)
    return learned.LoopSpec(n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0, hstep=-0.1, tilt_deg=1.0)


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


def run_b200(args, world, rank, local):
    import torch

    from mammos_mumag import _native, learned

    if _native.device_count() < 1:
        raise RuntimeError("no sm_100 GPU visible")
    torch.cuda.set_device(local)
    X, T, tag, krn, m0, hdir, sweep, desc = workload(args.workload, seed=rank)
    sp = _native.solver_params(hdir=hdir)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    nfs_expected = int(abs(sweep["hfinal"] - sweep["hstart"]) / abs(sweep["hstep"])) + 1
    if sweep.get("max_steps"):
        nfs_expected = min(nfs_expected, sweep["max_steps"])
    sw = (sweep["hstart"], sweep["hfinal"], sweep["hstep"], sweep["mstep"], sweep["mfinal"])
    mx = sweep.get("max_steps", 0)
    use_learned = args.workload != "single" and not args.no_learned
    headline = "learned_mixed" if use_learned else "fp64"

    # the learned warm start's network: trained once at set-up (untimed) on plain loops of
    # other seeds of the workload's mesh family
    model, train_info = None, None
    if use_learned:
        spec = loop_spec(args.workload)
        nseed = 2 if args.workload == "large" else 4
        t0 = time.perf_counter()
        feats, targets = learned.collect([1000 + 10 * rank + q for q in range(nseed)], spec, samples=50000,
                                         device=local)
        t1 = time.perf_counter()
        model, loss = learned.train(feats, targets, epochs=30, device=local)
        train_info = {"samples": int(len(targets)), "training_meshes": nseed, "collect_s": t1 - t0,
                      "train_s": time.perf_counter() - t1, "loss_rel": loss}

    def make_mesh(prec, warm):
        msh = _native.Mesh(X, T, tag, krn, device=local, precision=prec)
        if warm == _native.WARM_LEARNED:
            msh.set_warm_start(warm, model)
        msh.set_state(m0, None, m0)
        msh.autotune(sp)  # launch shape (set-up, untimed)
        return msh

    def timed(msh, clk_index=None):
        """W untimed sweeps, then K sweeps timed with CUDA events on the library's stream,
        the L2 flushed before each.  Returns (ms over ranks, field steps, step dicts, rows)."""
        for _ in range(args.warmup):
            msh.set_state(m0, None, m0)
            msh.loop(*sw, sp, max_steps=mx)
        total_ms, nfs, steps_all, rows = 0.0, 0, [], None
        dist_barrier(world)
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.fill_(1.0)  # L2 flush between timed sweeps (256 MB > 126 MB L2)
            torch.cuda.synchronize()
            msh.set_state(m0, None, m0)
            msh.timer_start()
            rows, steps = msh.loop(*sw, sp, max_steps=mx)
            total_ms += msh.timer_stop()
            nfs += len(rows)
            steps_all += steps
        torch.cuda.synchronize()
        dist_barrier(world)
        return dist_max(total_ms, world), nfs, steps_all, rows

    paths = {"fp64": (_native.PREC_FP64, _native.WARM_PREVIOUS)}
    if not args.no_mixed:
        paths["mixed"] = (_native.PREC_MIXED, _native.WARM_PREVIOUS)
    if use_learned:
        paths["learned_mixed"] = (_native.PREC_MIXED, _native.WARM_LEARNED)
    variants, raw = {}, {}
    clk = None
    for name, (prec, warm) in paths.items():
        msh = make_mesh(prec, warm)
        info = msh.info()
        if name == headline:
            with ClockSampler(local) as clk:
                res = timed(msh)
        else:
            res = timed(msh)
        msh.close()
        t_ms, nfs, st, rows = res
        evals = sum(x["evals"] for x in st)
        hc, mr = hc_mr(rows)
        raw[name] = (t_ms, nfs, st, rows, info)
        variants[name] = {"value": nfs * world / (t_ms * 1e-3),
                          "pcg_iters_per_solve": sum(x["pcg_iters"] for x in st) / max(1, evals),
                          "hc_T": hc, "mr_T": mr, "grid_ctas": info["grid_ctas"], "pcg_variant": info["pcg_variant"]}
    ref = variants["fp64"]
    for name, v in variants.items():
        if name == "fp64":
            continue
        v["speedup_vs_fp64"] = v["value"] / ref["value"]
        v["pcg_per_solve_vs_fp64"] = v["pcg_iters_per_solve"] / ref["pcg_iters_per_solve"]
        v["dHc_rel"] = (abs(v["hc_T"] - ref["hc_T"]) / ref["hc_T"]
                        if np.isfinite(ref["hc_T"]) and np.isfinite(v["hc_T"]) else None)
        v["dMr_rel"] = (abs(v["mr_T"] - ref["mr_T"]) / abs(ref["mr_T"])
                        if np.isfinite(ref["mr_T"]) and np.isfinite(v["mr_T"]) else None)
    t_max, nfs, steps_all, rows, info = raw[headline]
    value = variants[headline]["value"]
    launches = len(steps_all)
    kernel_ms = sum(st["device_ms"] for st in steps_all)
    Z, N = info["nnz"], info["nodes"]
    s_pcg = 4 if headline != "fp64" else 8
    ab = algorithmic_bytes(steps_all, Z, N, s_pcg=s_pcg)
    achieved = ab / (kernel_ms * 1e-3) / 1e9  # GB/s over the kernel's own launch durations
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    ratio = TRAFFIC_PER_ALGORITHMIC_BYTE.get((args.workload, headline))
    traffic = ratio * ab / launches if ratio is not None else None
    prec_h, warm_h = paths[headline]
    # e2e: the public API from host buffers (pinned), every step: mesh build + upload,
    # warm-start set-up, state upload, sweep, result read-back
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in
           (("X", X), ("T", np.asarray(T, np.int32)), ("tag", np.asarray(tag, np.int32)), ("m0", m0))}
    h2d = sum(t.numel() * t.element_size() for t in pin.values()) + 48 * len(krn)
    e2e_t, e2e_n = 0.0, 0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with _native.Mesh(pin["X"].numpy(), pin["T"].numpy(), pin["tag"].numpy(), krn, device=local,
                          precision=prec_h) as mm:
            if warm_h == _native.WARM_LEARNED:
                mm.set_warm_start(warm_h, model)
            mm.set_state(pin["m0"].numpy(), None, pin["m0"].numpy())
            mm.autotune(sp)  # cached for this mesh shape: no timing runs after the first
            r2, _ = mm.loop(*sw, sp, max_steps=mx)
            mfin, _, _ = mm.get_state()
        e2e_t += time.perf_counter() - t0
        e2e_n += len(r2)
    d2h = 32 * nfs_expected + mfin.nbytes
    e2e_t = dist_max(e2e_t, world)
    if rank == 0:
        cpu = None
        if world == 1 and args.workload != "large":
            v, dt, n = cpu_sample(args.workload, 12)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"first {n} field steps of the sweep ({dt:.1f} s), NumPy/SciPy oracle, single thread"}
        evals = sum(st["evals"] for st in steps_all)
        pcg = sum(st["pcg_iters"] for st in steps_all)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if headline == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": desc, "path": headline,
                       "precision": "fp64" if prec_h == _native.PREC_FP64 else
                       "mixed (FP32 operator planes and inner PCG, FP64 refinement, reductions, energies)",
                       "warm_start": "learned" if warm_h == _native.WARM_LEARNED else "previous u (reference)",
                       "parallelism": f"replicas x{world}",
                       "l2": "256 MB buffer written between timed sweeps (L2 flush)",
                       "grid_ctas": info["grid_ctas"], "block_threads": info["block_threads"],
                       "pcg_variant": info["pcg_variant"]},
            "pcg_iters_per_solve": pcg / max(1, evals),
            "variants": variants,
            "learned_training": train_info,
            "field_steps_per_sweep": nfs // args.steps,
            "hc_T": variants[headline]["hc_T"], "mr_T": variants[headline]["mr_T"],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": ("DRAM bytes per algorithmic byte of one ncu-captured field-step "
                                            "launch of this path, scaled to the average launch")
                         if traffic is not None else None,
                         "kernel": f"k_solve (persistent field step, {headline})",
                         "algorithmic_bytes_per_launch": ab / launches,
                         "avg_launch_ms": kernel_ms / launches,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_n * world / e2e_t, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
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
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["multigrain", "single", "large", "batch"], default="multigrain")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision variant")
    ap.add_argument("--ref-procs", type=int, default=1,
                    help="reference arm: independent replica processes (0: one per usable host core); the "
                         "default 1 times the workload as configured, one sweep")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned warm start (headline = the plain FP64 path)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
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
