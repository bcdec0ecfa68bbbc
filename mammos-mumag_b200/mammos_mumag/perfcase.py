"""Small, fixed launch sequences of the library's kernels, for profilers and timing.

    python -m mammos_mumag.perfcase field-step [--workload multigrain|large] [--precision fp64|mixed]
                                               [--grid N] [--ctas-per-sm 2|3] [--pcg-variant 1|2]
                                               [--coarse BOX_NODES] [--learned]
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
    mt = sub.add_parser("mlp-train")
    mt.add_argument("--samples", type=int, default=16384)
    mt.add_argument("--epochs", type=int, default=2)
    mp = sub.add_parser("mlp-predict")
    mp.add_argument("--rows", type=int, default=531441)
    args = ap.parse_args(argv)
    return {"field-step": field_step, "mlp-train": mlp_train, "mlp-predict": mlp_predict}[args.case](args)


if __name__ == "__main__":
    sys.exit(main())
