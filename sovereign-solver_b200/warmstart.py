"""Learned warm start for a parametric LP family (b = b0 + B_b theta,
c = c0 + B_c theta over one matrix).

1. Training data: the family's training instances solved by the batched
   engine (``Engine.solve_batch``, one CUDA-graph launch per chunk).
2. Basis: the top ``rank`` principal directions of the primal solutions and of
   the dual solutions (host SVD of the centred solution matrices; set-up, not
   on the solve path).
3. Network: ``mlp.Mlp`` (tensor-core BF16 GEMMs, FP32 accumulation, Adam on
   the device) maps theta / theta_std to the standardised basis coefficients.
4. Use: the predicted point is a candidate start (x0, y0). It is kept only if
   its relative KKT residual (PDLP's l2 measure, evaluated on the device by
   ``Engine.start_kkt``) is below the cold start's; otherwise the instance
   starts cold. Plain PDHG is
   therefore both the fallback and the gate, and every solve is held to the
   same termination tolerance.
5. Fallback at run time (``solve_family_with_fallback``): a warm-started
   solve gets as many iterations as the most any training solve of the family
   needed from the cold start (``LearnedWarmStart.budget``); an instance that
   is not optimal by then is solved again from the cold start with the full
   cap, and its result counts the iterations of both attempts.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace

import numpy as np

from . import lpgen
from .mlp import Mlp
from .pdhg import Engine, PdhgOptions, PdhgResult


def relative_kkt(p, r: PdhgResult) -> float:
    """max(primal/(1+|b|inf), dual/(1+|c|inf), gap) of a reported point."""
    fin = lambda a: a[np.isfinite(a)]  # noqa: E731
    bnorm = max(np.max(np.abs(fin(p.row_lo)), initial=0.0), np.max(np.abs(fin(p.row_hi)),
                                                                       initial=0.0))
    cnorm = float(np.max(np.abs(p.c), initial=0.0))
    return max(r.primal_infeasibility / (1.0 + bnorm), r.dual_infeasibility / (1.0 + cnorm),
               r.duality_gap)


def solve_family(engine: Engine, problems: list, opt: PdhgOptions, x0s=None, y0s=None,
                 chunk: int = 256) -> list[PdhgResult]:
    """Batched solves of a list of LPs, `chunk` instances per batch."""
    out = []
    for i in range(0, len(problems), chunk):
        engine.load_batch(problems[i:i + chunk])
        xs = None if x0s is None else list(x0s[i:i + chunk])
        ys = None if y0s is None else list(y0s[i:i + chunk])
        out.extend(engine.solve_batch(opt, x0=xs, y0=ys))
    return out


def solve_family_with_fallback(engine: Engine, problems: list, opt: PdhgOptions, x0s, y0s,
                               budget: int, chunk: int = 256) -> list[PdhgResult]:
    """Batched solves from the starts (x0s, y0s) with at most `budget`
    iterations each; the instances that end without an optimal status are
    solved again, batched, from the cold start with `opt`'s own cap. Their
    results report the iterations of both attempts. Returns one result per
    problem, in order."""
    if x0s is None or budget <= 0 or budget >= opt.max_iterations:
        return solve_family(engine, problems, opt, x0s, y0s, chunk)
    warm = solve_family(engine, problems, replace(opt, max_iterations=budget), x0s, y0s, chunk)
    redo = [i for i, r in enumerate(warm) if r.status != "optimal"]
    if redo:
        cold = solve_family(engine, [problems[i] for i in redo], opt, chunk=chunk)
        for i, r in zip(redo, cold):
            r.iterations += warm[i].iterations
            warm[i] = r
    return warm


@dataclass
class FitReport:
    samples: int
    rank: int
    explained_primal: float
    explained_dual: float
    losses: np.ndarray


class LearnedWarmStart:
    def __init__(self, family: lpgen.ParametricFamily, rank: int = 256, hidden: int = 512,
                 device: int = 0) -> None:
        self.family = family
        self.rank = rank
        self.hidden = hidden
        self.device = device
        self.net: Mlp | None = None
        self.budget = 0  # iteration budget of a warm solve, set by fit()

    # ---- basis and network ----------------------------------------------------

    @staticmethod
    def _basis(sol: np.ndarray, rank: int):
        mean = sol.mean(axis=0)
        u, s, vt = np.linalg.svd(sol - mean, full_matrices=False)
        total = float(np.sum(s * s)) or 1.0
        return mean, vt[:rank].T, s[:rank], float(np.sum(s[:rank] ** 2) / total)

    def fit(self, thetas: np.ndarray, results: list[PdhgResult], epochs: int = 300,
            batch: int = 64, lr: float = 1e-3, seed: int = 0, val_frac: float = 0.15,
            rounds: int = 10) -> FitReport:
        """Basis + network from solved training instances (optimal ones only).
        A `val_frac` share is held out: the network trains in `rounds` rounds of
        epochs / rounds epochs and keeps the parameters of the round with the
        lowest validation loss."""
        keep = [i for i, r in enumerate(results) if r.status == "optimal"]
        # the warm solves' iteration budget: the most any optimal training
        # solve of the family took from the cold start
        self.budget = max((results[i].iterations for i in keep), default=0)
        th = np.asarray(thetas)[keep]
        xs = np.stack([results[i].primal for i in keep])
        ys = np.stack([results[i].dual for i in keep])
        r = min(self.rank, len(keep) - 1)
        r -= r % 4  # 2 r outputs: a multiple of 8
        if r < 4:
            raise ValueError("too few solved training instances for a basis")
        self.mx, self.Ux, sx, ex = self._basis(xs, r)
        self.my, self.Uy, sy, ey = self._basis(ys, r)
        cx = (xs - self.mx) @ self.Ux
        cy = (ys - self.my) @ self.Uy
        coef = np.hstack([cx, cy])
        self.cscale = coef.std(axis=0) + 1e-12
        target = coef / self.cscale
        self.r = r
        n_in = self.family.n_params
        mb = max(8, min(512, (batch + 7) // 8 * 8))
        if self.net is not None:
            self.net.close()
        self.net = Mlp(n_in, self.hidden, 2 * r, max_batch=max(mb, 256), device=self.device)
        rng = np.random.default_rng(seed)
        w1 = rng.standard_normal((self.hidden, n_in)) * math.sqrt(2.0 / n_in)
        w2 = rng.standard_normal((self.hidden, self.hidden)) * math.sqrt(2.0 / self.hidden)
        w3 = rng.standard_normal((2 * r, self.hidden)) * math.sqrt(1.0 / self.hidden)
        self.net.set_params(np.concatenate([w1.ravel(), np.zeros(self.hidden), w2.ravel(),
                                            np.zeros(self.hidden), w3.ravel(),
                                            np.zeros(2 * r)]))
        x_in = th / self.family.theta_std
        perm = np.random.default_rng(seed + 7).permutation(len(keep))
        n_val = int(round(val_frac * len(keep))) if rounds > 1 else 0
        val, tr = perm[:n_val], perm[n_val:]
        steps_batch = min(mb, (len(tr) // 8) * 8)
        per = max(1, epochs // max(rounds, 1))
        losses, best, best_params = [], np.inf, None
        for rnd in range(max(rounds, 1)):
            losses.extend(self.net.train(x_in[tr], target[tr], epochs=per, batch=steps_batch,
                                         lr=lr, seed=seed + rnd))
            if n_val == 0:
                continue
            pv = self.net.forward(x_in[val])
            vl = float(np.mean((pv - target[val]) ** 2))
            if vl < best:
                best, best_params = vl, self.net.get_params()
        if best_params is not None:
            self.net.set_params(best_params)
        self.val_loss = best
        return FitReport(len(keep), r, ex, ey, np.asarray(losses))

    def predict(self, thetas: np.ndarray):
        """Candidate starts (x0, y0) in original units, one row per theta."""
        out = self.net.forward(np.asarray(thetas) / self.family.theta_std) * self.cscale
        x0 = self.mx + out[:, : self.r] @ self.Ux.T
        y0 = self.my + out[:, self.r:] @ self.Uy.T
        # duals of one-sided rows onto their sign (a wrong sign makes the dual
        # objective -inf in the result's gap): <= rows y <= 0, >= rows y >= 0
        base = self.family.base
        upper_only = ~np.isfinite(base.row_lo) & np.isfinite(base.row_hi)
        lower_only = np.isfinite(base.row_lo) & ~np.isfinite(base.row_hi)
        y0[:, upper_only] = np.minimum(y0[:, upper_only], 0.0)
        y0[:, lower_only] = np.maximum(y0[:, lower_only], 0.0)
        return x0, y0

    # ---- gated starts ----------------------------------------------------------

    def starts(self, engine: Engine, problems: list, thetas: np.ndarray, opt: PdhgOptions,
               chunk: int = 256):
        """Per instance the predicted start where its relative KKT residual is
        below the cold start's, else the cold start (x = 0 projected, y = 0).
        Returns (x0s, y0s, used, kkt_warm, kkt_cold)."""
        x0, y0 = self.predict(thetas)
        kw, kc = [], []
        for i in range(0, len(problems), chunk):
            engine.load_batch(problems[i:i + chunk])
            kw.append(engine.start_kkt(list(x0[i:i + chunk]), list(y0[i:i + chunk])))
            kc.append(engine.start_kkt())
        kw, kc = np.concatenate(kw), np.concatenate(kc)
        used = kw < kc
        xs = [x0[i] if used[i] else np.zeros(p.n) for i, p in enumerate(problems)]
        ys = [y0[i] if used[i] else np.zeros(p.m) for i, p in enumerate(problems)]
        return xs, ys, used, kw, kc
