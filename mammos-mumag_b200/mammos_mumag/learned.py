"""Learned warm start of the magnetostatic Poisson solve: training data, training, evaluation.

The reference starts every Poisson PCG from the previous potential
(``scripts/solvers.py:221-231``, ``x0=u``).  This module builds the learned alternative and
measures it against that start and against a zero start:

1. ``collect``: run plain-solver hysteresis loops on seeded multigrain meshes with sample
   recording on (``Mesh.record_samples``): at a hash-selected fraction of the (node, solve)
   pairs the library stores the node's 16 features at the warm start and, after the solve,
   the target ``(u - u_prev)/sigma``.
2. ``train``: fit the network (``Model``) with the library's tensor-core training kernels.
3. ``compare``: run the same loops on held-out seeds with each warm start and report PCG
   iterations per solve, field steps per second and the loops' Hc/Mr.

Every solve still runs to the reference's tolerance, so the loops' results agree between
warm starts to within that tolerance's effect on the minimiser.
"""

from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import _native, synthetic

WARM_NAMES = {_native.WARM_PREVIOUS: "previous", _native.WARM_ZERO: "zero", _native.WARM_LEARNED: "learned"}


@dataclasses.dataclass
class LoopSpec:
    """A seeded multigrain loop: mesh (cube edge L nm, n^3 cells), grains, field sweep."""

    n: int = 16
    L: float = 20.0
    grains: int = 4
    cone_deg: float = 15.0
    gb: float = 2.0
    hstart: float = 8.0
    hfinal: float = -8.0
    hstep: float = -0.2
    mfinal: float = -2.0
    tilt_deg: float = 1.0
    precision: int = _native.PREC_FP64
    max_steps: int = 0  # > 0: only the first max_steps field steps

    @property
    def steps(self) -> int:
        n = int(abs(self.hfinal - self.hstart) / abs(self.hstep)) + 1
        return min(n, self.max_steps) if self.max_steps > 0 else n

    def hdir(self):
        t = np.radians(self.tilt_deg)
        return [float(np.sin(t)), 0.0, float(np.cos(t))]

    def mesh(self, seed: int, device: int = 0, precision: int | None = None):
        X, T, tag, krn, m0 = synthetic.multigrain(n=self.n, L=self.L, grains=self.grains, cone_deg=self.cone_deg,
                                                  gb=self.gb, seed=seed)
        prec = self.precision if precision is None else precision
        M = _native.Mesh(X, T, tag, krn, precision=prec, device=device)
        return M, m0

    def run(self, M, m0, max_steps: int = 0):
        sp = _native.solver_params(hdir=self.hdir())
        M.set_state(m0, np.zeros(M.N), m0)
        mx = max_steps if max_steps > 0 else self.max_steps
        return M.loop(self.hstart, self.hfinal, self.hstep, abs(self.hstep), self.mfinal, sp, max_steps=mx)


def collect(seeds, spec: LoopSpec | None = None, samples: int = 50000, device: int = 0, rng_seed: int = 0,
            evals_per_step: int = 30):
    """``(feats [k,16], targets [k])`` from plain (previous-u) loops on ``seeds``; about
    ``samples`` in total, spread uniformly over each loop's solves."""
    spec = spec or LoopSpec()
    rng = np.random.default_rng(rng_seed)
    per_mesh = int(np.ceil(samples / len(seeds)))
    F, Tg = [], []
    for s in seeds:
        M, m0 = spec.mesh(s, device)
        with M:
            candidates = M.N * spec.steps * evals_per_step
            stride = max(1, candidates // (2 * per_mesh))
            M.record_samples(8 * per_mesh, stride=stride, seed=int(s) * 7919 + 1)
            spec.run(M, m0)
            f, t, _ = M.read_samples()
            M.record_samples(0)
        if len(t) > per_mesh:
            keep = rng.choice(len(t), per_mesh, replace=False)
            f, t = f[keep], t[keep]
        F.append(f)
        Tg.append(t)
    return np.concatenate(F), np.concatenate(Tg)


def train(feats, targets, epochs: int = 30, batch: int = 256, lr: float = 1e-3, seed: int = 0, device: int = 0):
    """A trained ``Model`` (normalisation fitted to the data) and its final training loss."""
    model = _native.Model(device=device, seed=seed)
    model.fit_normalization(feats, targets)
    loss = model.train(feats, targets, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return model, loss


def hc_mr(rows):
    """Coercive field and remanence of a loop's rows (``hysteresis.coercivity_remanence``)."""
    from .hysteresis import coercivity_remanence

    return coercivity_remanence(rows)


def compare(model, seeds, spec: LoopSpec | None = None, device: int = 0, modes=(0, 1, 2), max_steps: int = 0):
    """Per warm start: PCG iterations per solve (summed over the seeds' loops), field steps
    per second (device time), and per-seed rows / Hc / Mr."""
    spec = spec or LoopSpec()
    out = {}
    for mode in modes:
        pcg = evals = steps = 0
        ms = 0.0
        per_seed = []
        for s in seeds:
            M, m0 = spec.mesh(s, device)
            with M:
                M.set_warm_start(mode, model if mode == _native.WARM_LEARNED else None)
                M.timer_start()
                rows, st = spec.run(M, m0, max_steps=max_steps)
                ms += M.timer_stop()
            pcg += sum(d["pcg_iters"] for d in st)
            evals += sum(d["evals"] for d in st)
            steps += len(st)
            per_seed.append({"seed": int(s), "rows": rows, "hc_mr": hc_mr(rows)})
        out[WARM_NAMES[mode]] = {
            "pcg_per_solve": pcg / max(1, evals),
            "pcg_iters": int(pcg),
            "solves": int(evals),
            "steps": int(steps),
            "steps_per_s": steps / (ms / 1e3) if ms > 0 else float("nan"),
            "per_seed": per_seed,
        }
    return out


def experiment(train_seeds=range(16), test_seeds=range(100, 104), spec: LoopSpec | None = None,
               samples: int = 50000, epochs: int = 30, device: int = 0):
    """Collect, train, compare; returns a summary dict (no per-seed rows)."""
    spec = spec or LoopSpec()
    t0 = time.perf_counter()
    feats, targets = collect(list(train_seeds), spec, samples, device)
    t1 = time.perf_counter()
    model, loss = train(feats, targets, epochs=epochs, device=device)
    t2 = time.perf_counter()
    res = compare(model, list(test_seeds), spec, device)
    summary = {
        "samples": int(len(targets)),
        "collect_s": t1 - t0,
        "train_s": t2 - t1,
        "train_loss": loss,  # mean squared error over the targets' mean square (1 = predicting 0)
    }
    for k, v in res.items():
        summary[k] = {kk: vv for kk, vv in v.items() if kk != "per_seed"}
        summary[k]["hc_mr"] = [p["hc_mr"] for p in v["per_seed"]]
    return model, summary
