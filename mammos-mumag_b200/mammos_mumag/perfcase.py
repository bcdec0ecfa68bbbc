"""Small, fixed launch sequences of the library's kernels, for profilers and timing.

    python -m mammos_mumag.perfcase field-step [--workload multigrain|large] [--precision fp64|mixed]
                                               [--grid N] [--ctas-per-sm 2|3] [--pcg-variant 1|2]
                                               [--coarse BOX_NODES] [--learned]
    python -m mammos_mumag.perfcase poisson-solve [--workload multigrain|large] [--precision fp64|mixed]
                                                  [--grid N] [--ctas-per-sm 2|3] [--pcg-variant 1|2]
                                                  [--coarse BOX_NODES]
    python -m mammos_mumag.perfcase phase-timers [--workload multigrain|large] [--precision fp64|mixed]
                                                 [--grid N] [--ctas-per-sm 2|3] [--pcg-variant 1|2]
                                                 [--coarse BOX_NODES] [--from-step K] [--steps S]
    python -m mammos_mumag.perfcase minv [--workload multigrain|large] [--precision fp64|mixed]
                                         [--grid N] [--ctas-per-sm 2|3] [--coarse BOX_NODES]
    python -m mammos_mumag.perfcase mlp-train [--samples N] [--epochs E]
    python -m mammos_mumag.perfcase mlp-predict [--rows N]

``field-step``: builds the workload's mesh with a fixed launch shape (no autotuning, so the
launch sequence is known), then runs two field steps (``mm_minimize``) from the seeded
initial state: the first is a warm-up, the second the measured launch.  Kernel launches in
order: the assembly kernels, then ``k_solve`` twice.  Prints the second launch's device time
and work counters.  With ``--learned`` the mesh uses the learned warm start: first a
network is trained on samples recorded from the first 10 field steps of another seed of the
same family (10 ``k_solve`` launches and the training kernels), so the measured launch is
the 12th ``k_solve`` launch.

``poisson-solve``: the same mesh and launch shape; one field step from the seeded initial
state (``k_solve`` launch 1), then two energy evaluations (``mm_energy_grad``, ``k_solve``
launches 2 and 3) whose Poisson solves start from u = 0, so those launches are dominated by
the PCG iterations.  Prints the last launch's PCG iterations and the per-iteration device
time.

``phase-timers``: the per-CTA phase timers of the persistent kernel (MUMAG_PROFILE, set by
this case before the mesh is built) over S field steps of the workload's sweep from field
step K (the steps before K run first, untimed): device time, work counters and the mean per
CTA of the PCG row phases, the reductions (before, waiting at and after the grid barrier),
the coarse update, whole Poisson solves, M_inv and the evaluations.

``minv``: the same mesh and launch shape; one field step from the seeded initial state, one
energy evaluation at a field 1 T lower, then the M_inv preconditioner (``mm_apply_minv``, one
``k_solve`` launch each, truncated CG of up to 10 iterations) applied three times to that
evaluation's gradient: launches 3 to 5 are M_inv alone.

``mlp-predict``: the network on N seeded feature rows (``k_predict``), twice.

``mlp-train``: trains the warm-start network for a few epochs on seeded synthetic samples
(batches of 256 rows): per batch ``k_gather``, ``k_fwd``, ``k_bwd``, three ``k_wgrad``, three
``k_bsum``, ``k_adam``, ``k_publish``.

Workloads (as in ``bench.py``): multigrain = 80 nm cube, 32^3 x 6 tets, 8 grains + 2 nm
grain-boundary phase; large = 200 nm cube, 80^3 x 6 tets (3,072,000 tets), 27 grains.
"""

from __future__ import annotations

import argparse
import sys

import numpy as np

from . import _native, synthetic


def field_step(args) -> int:
    if args.workload == "large":
        X, T, tag, krn, m0 = synthetic.multigrain(n=80, L=200.0, grains=27, cone_deg=20.0, gb=2.0, seed=0)
        hdir, h0, dh = [0.0, 0.0, 1.0], 8.0, -0.05
    else:
        X, T, tag, krn, m0 = synthetic.multigrain(n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0, seed=0)
        d = np.radians(1.0)
        hdir, h0, dh = [float(np.sin(d)), 0.0, float(np.cos(d))], 8.0, -0.1
    prec = _native.PREC_MIXED if args.precision == "mixed" else _native.PREC_FP64
    sp = _native.solver_params(hdir=hdir)
    model = None
    if args.learned:
        from . import learned

        if args.workload == "large":
            spec = learned.LoopSpec(n=80, L=200.0, grains=27, cone_deg=20.0, gb=2.0, hstep=-0.05, tilt_deg=0.0,
                                    max_steps=10)
        else:
            spec = learned.LoopSpec(n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0, hstep=-0.1, tilt_deg=1.0,
                                    max_steps=10)
        feats, targets = learned.collect([1], spec, samples=20000, evals_per_step=10)
        model, _ = learned.train(feats, targets, epochs=5)
    with _native.Mesh(X, T, tag, krn, precision=prec, grid_ctas=args.grid, ctas_per_sm=args.ctas_per_sm,
                      pcg_variant=args.pcg_variant, coarse_box_nodes=args.coarse) as M:
        if model is not None:
            M.set_warm_start(_native.WARM_LEARNED, model)
        M.set_state(m0, None, m0)
        M.minimize(h0, sp)
        r = M.minimize(h0 + dh, sp)
        info = M.info()
    print(f"field step: {args.workload} {args.precision} grid {info['grid_ctas']} x {info['block_threads']} "
          f"(build {info['kernel_ctas_per_sm']} CTAs/SM, PCG arrangement {info['pcg_variant']}): "
          f"{r['device_ms']:.3f} ms, PCG iterations {r['pcg_iters']}, evaluations {r['evals']}, "
          f"M_inv iterations {r['minv_iters']}, NCG iterations {r['ncg_iters']}"
          + (f", two-level preconditioner ({info['coarse_boxes']} boxes)" if info["coarse_boxes"] else "")
          + (", learned warm start" if model is not None else ""))
    if model is not None:
        model.close()
    return 0


def _workload_mesh(args):
    if args.workload == "large":
        X, T, tag, krn, m0 = synthetic.multigrain(n=80, L=200.0, grains=27, cone_deg=20.0, gb=2.0, seed=0)
        hdir, h0 = [0.0, 0.0, 1.0], 8.0
    else:
        X, T, tag, krn, m0 = synthetic.multigrain(n=32, L=80.0, grains=8, cone_deg=15.0, gb=2.0, seed=0)
        d = np.radians(1.0)
        hdir, h0 = [float(np.sin(d)), 0.0, float(np.cos(d))], 8.0
    return X, T, tag, krn, m0, hdir, h0


def poisson_solve(args) -> int:
    X, T, tag, krn, m0, hdir, h0 = _workload_mesh(args)
    prec = _native.PREC_MIXED if args.precision == "mixed" else _native.PREC_FP64
    sp = _native.solver_params(hdir=hdir)
    with _native.Mesh(X, T, tag, krn, precision=prec, grid_ctas=args.grid, ctas_per_sm=args.ctas_per_sm,
                      pcg_variant=args.pcg_variant, coarse_box_nodes=args.coarse) as M:
        M.set_state(m0, None, m0)
        M.minimize(h0, sp)
        m, u, _ = M.get_state()
        zero = np.zeros_like(u)
        for _ in range(2):
            M.set_state(m, zero, m0)
            M.timer_start()
            _, _, iters = M.energy_grad(h0, sp)
            ms = M.timer_stop()
        info = M.info()
    print(f"poisson-solve: {args.workload} {args.precision} grid {info['grid_ctas']} x {info['block_threads']} "
          f"(build {info['kernel_ctas_per_sm']} CTAs/SM, PCG arrangement {info['pcg_variant']}"
          + (f", two-level preconditioner ({info['coarse_boxes']} boxes)" if info["coarse_boxes"] else "")
          + f"): {iters} PCG iterations, {ms:.3f} ms with the state upload, {1e3 * ms / max(iters, 1):.1f} us per iteration")
    return 0


def phase_timers(args) -> int:
    import os

    os.environ["MUMAG_PROFILE"] = "1"
    X, T, tag, krn, m0, hdir, h0 = _workload_mesh(args)
    dh = -0.05 if args.workload == "large" else -0.1
    prec = _native.PREC_MIXED if args.precision == "mixed" else _native.PREC_FP64
    sp = _native.solver_params(hdir=hdir)
    with _native.Mesh(X, T, tag, krn, precision=prec, grid_ctas=args.grid, ctas_per_sm=args.ctas_per_sm,
                      pcg_variant=args.pcg_variant, coarse_box_nodes=args.coarse) as M:
        M.set_state(m0, None, m0)
        h = h0
        for _ in range(args.from_step):
            M.minimize(h, sp)
            h += dh
        M.profile()
        tot = np.zeros(12)
        cnt = dict.fromkeys(("device_ms", "evals", "pcg_iters", "minv_iters", "ncg_iters", "barriers"), 0.0)
        for _ in range(args.steps):
            r = M.minimize(h, sp)
            h += dh
            tot += M.profile().astype(float).mean(axis=0) / 1e6
            for k in cnt:
                cnt[k] += r[k]
        info = M.info()
    names = ("PCG row phases", "reduction before barrier", "barrier wait", "reduction after barrier",
             "Poisson solves", "M_inv", "evaluations (solves included)", "launches", "", "coarse update")
    print(f"phase-timers: {args.workload} {args.precision} grid {info['grid_ctas']} x {info['block_threads']}"
          + (f", two-level preconditioner ({info['coarse_boxes']} boxes)" if info["coarse_boxes"] else "")
          + f", field steps {args.from_step}..{args.from_step + args.steps - 1}")
    print("  counters: " + ", ".join(f"{k} {v:.0f}" for k, v in cnt.items()))
    for i, nm in enumerate(names):
        if nm:
            print(f"  {nm:32s} {tot[i]:9.1f} ms per CTA")
    print(f"  per PCG iteration: {1e3 * tot[4] / max(cnt['pcg_iters'], 1):.1f} us in Poisson solves; per M_inv "
          f"iteration: {1e3 * tot[5] / max(cnt['minv_iters'], 1):.1f} us")
    return 0


def minv(args) -> int:
    X, T, tag, krn, m0, hdir, h0 = _workload_mesh(args)
    prec = _native.PREC_MIXED if args.precision == "mixed" else _native.PREC_FP64
    sp = _native.solver_params(hdir=hdir)
    with _native.Mesh(X, T, tag, krn, precision=prec, grid_ctas=args.grid, ctas_per_sm=args.ctas_per_sm,
                      pcg_variant=args.pcg_variant, coarse_box_nodes=args.coarse) as M:
        M.set_state(m0, None, m0)
        M.minimize(h0, sp)
        _, g, _ = M.energy_grad(h0 - 1.0, sp)
        for _ in range(3):
            M.timer_start()
            _, iters = M.apply_minv(g, sp)
            ms = M.timer_stop()
        info = M.info()
    print(f"minv: {args.workload} {args.precision} grid {info['grid_ctas']} x {info['block_threads']} "
          f"(build {info['kernel_ctas_per_sm']} CTAs/SM): {iters} truncated-CG iterations, {ms:.3f} ms with the "
          f"vector transfers")
    return 0


def mlp_train(args) -> int:
    rng = np.random.default_rng(0)
    feats = rng.standard_normal((args.samples, _native.MLP_FEATURES)).astype(np.float32)
    target = (np.tanh(feats[:, 0] * feats[:, 3]) + 0.3 * feats[:, 12]).astype(np.float32)
    with _native.Model(seed=0) as model:
        model.fit_normalization(feats, target)
        loss = model.train(feats, target, epochs=args.epochs, batch=256, lr=1e-3, seed=0)
    print(f"mlp-train: {args.samples} samples, {args.epochs} epochs, final loss {loss:.4f}")
    return 0


def mlp_predict(args) -> int:
    rng = np.random.default_rng(0)
    feats = rng.standard_normal((args.rows, _native.MLP_FEATURES)).astype(np.float32)
    with _native.Model(seed=0) as model:
        y = model.predict(feats)
        y = model.predict(feats)
    print(f"mlp-predict: {args.rows} rows, mean output {float(np.mean(y)):.6f}")
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="case", required=True)
    fs = sub.add_parser("field-step")
    fs.add_argument("--workload", choices=["multigrain", "large"], default="multigrain")
    fs.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    fs.add_argument("--grid", type=int, default=0, help="CTAs (0: the size-based default)")
    fs.add_argument("--ctas-per-sm", type=int, choices=[0, 2, 3], default=0)
    fs.add_argument("--pcg-variant", type=int, choices=[0, 1, 2], default=0)
    fs.add_argument("--coarse", type=int, default=0,
                    help="two-level Poisson preconditioner with boxes of about this many nodes (0: Jacobi)")
    fs.add_argument("--learned", action="store_true", help="learned warm start (trains a network first)")
    ps = sub.add_parser("poisson-solve")
    ps.add_argument("--workload", choices=["multigrain", "large"], default="large")
    ps.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ps.add_argument("--grid", type=int, default=0, help="CTAs (0: the size-based default)")
    ps.add_argument("--ctas-per-sm", type=int, choices=[0, 2, 3], default=0)
    ps.add_argument("--pcg-variant", type=int, choices=[0, 1, 2], default=0)
    ps.add_argument("--coarse", type=int, default=0,
                    help="two-level Poisson preconditioner with boxes of about this many nodes (0: Jacobi)")
    pt = sub.add_parser("phase-timers")
    pt.add_argument("--workload", choices=["multigrain", "large"], default="large")
    pt.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    pt.add_argument("--grid", type=int, default=0, help="CTAs (0: the size-based default)")
    pt.add_argument("--ctas-per-sm", type=int, choices=[0, 2, 3], default=0)
    pt.add_argument("--pcg-variant", type=int, choices=[0, 1, 2], default=0)
    pt.add_argument("--coarse", type=int, default=0,
                    help="two-level Poisson preconditioner with boxes of about this many nodes (0: Jacobi)")
    pt.add_argument("--from-step", type=int, default=211)
    pt.add_argument("--steps", type=int, default=6)
    mi = sub.add_parser("minv")
    mi.add_argument("--workload", choices=["multigrain", "large"], default="large")
    mi.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    mi.add_argument("--grid", type=int, default=0, help="CTAs (0: the size-based default)")
    mi.add_argument("--ctas-per-sm", type=int, choices=[0, 2, 3], default=0)
    mi.add_argument("--pcg-variant", type=int, choices=[0, 1, 2], default=0)
    mi.add_argument("--coarse", type=int, default=0,
                    help="two-level Poisson preconditioner with boxes of about this many nodes (0: Jacobi)")
    mt = sub.add_parser("mlp-train")
    mt.add_argument("--samples", type=int, default=16384)
    mt.add_argument("--epochs", type=int, default=2)
    mp = sub.add_parser("mlp-predict")
    mp.add_argument("--rows", type=int, default=531441)
    args = ap.parse_args(argv)
    return {"field-step": field_step, "poisson-solve": poisson_solve, "phase-timers": phase_timers,
            "minv": minv, "mlp-train": mlp_train, "mlp-predict": mlp_predict}[args.case](args)


if __name__ == "__main__":
    sys.exit(main())
