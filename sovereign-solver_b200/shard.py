"""One batch of LPs, and the warm-start network's training, across GPUs.

One process per GPU (torch.distributed, NCCL on the GPU box; gloo in the CPU
tests). The reference solves independent LPs one per thread, each with its
own Backend (src/l1/race.cpp:123-129); here the unit of independence is the
instance of a batch:

* ``partition`` cuts a batch into one part per rank with balanced total
  nonzeros (the work of an iteration is about proportional to them), largest
  instance first onto the least loaded rank; each part keeps ascending
  instance order.
* ``solve_sharded`` has every rank solve its part with the batched engine (one
  CUDA-graph launch, no per-iteration collective: the instances never talk to
  each other) and gathers the results to rank 0 in instance order: one
  collective per batch.
* ``train_data_parallel`` trains the network data-parallel: each global
  mini-batch is split across the ranks, each rank takes the gradient of its
  slice on its own GPU (pdhg_mlp_gradients), one allreduce averages the
  gradient vector (0.56M floats for the 64 -> 512 -> 512 -> 512 network), and
  every replica applies the same Adam step (pdhg_mlp_adam_step), so the
  replicas stay identical.

Both take their per-rank work as callables, so the host logic runs the same
with the engine on a GPU and with stand-ins on the CPU.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def partition(weights: Sequence[float], world: int) -> list[list[int]]:
    """Instance indices per rank, balanced by total weight (nonzeros): the
    heaviest instances first, each onto the rank with the least weight so far
    (ties to the rank with fewer instances, then the lower rank); every part
    in ascending instance order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda k: (-w[k], k))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], len(parts[q]), q))
        parts[r].append(k)
        load[r] += float(w[k])
    return [sorted(p) for p in parts]


def solve_sharded(problems: Sequence, solve_part: Callable[[list], list], rank: int,
                  world: int, weights: Sequence[float] | None = None):
    """Rank `rank`'s part of the batch solved by `solve_part` (a list of
    problems -> a list of results in the same order); rank 0 returns every
    result in instance order, the others None."""
    if weights is None:
        weights = [p.nnz for p in problems]
    parts = partition(weights, world)
    mine = parts[rank]
    results = solve_part([problems[k] for k in mine]) if mine else []
    if len(results) != len(mine):
        raise RuntimeError("solve_part returned a different number of results")
    if world == 1:
        return list(results)
    import torch.distributed as dist
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, results)), gathered, dst=0)
    if rank != 0:
        return None
    out = [None] * len(problems)
    for pairs in gathered:
        for k, r in pairs:
            out[k] = r
    if any(r is None for r in out):
        raise RuntimeError("an instance was not solved by any rank")
    return out


def allreduce_mean(v: np.ndarray, world: int, device=None) -> np.ndarray:
    """The mean of `v` over all ranks (one allreduce of the whole vector)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float32))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return (t / world).cpu().numpy()


def train_data_parallel(x: np.ndarray, t: np.ndarray, epochs: int, batch: int,
                        grad_fn: Callable[[np.ndarray, np.ndarray], tuple],
                        step_fn: Callable[[np.ndarray], None], rank: int, world: int,
                        seed: int = 0, device=None) -> np.ndarray:
    """Data-parallel training. Every rank draws the same shuffled order of the
    samples (seeded), cuts each global mini-batch of `batch` rows (a multiple
    of 8 x world) into `world` equal slices, takes the gradient of its slice
    with grad_fn(x_slice, t_slice) -> (gradient, loss), averages gradient and
    loss over the ranks and applies step_fn(gradient). Returns the mean loss of
    each epoch (the same on every rank). With equal slices the averaged
    gradient is the gradient of the whole mini-batch's mean loss."""
    if batch % world != 0 or (batch // world) % 8 != 0:
        raise ValueError("batch must be a multiple of 8 x world")
    per = batch // world
    samples = x.shape[0]
    steps = samples // batch
    if steps < 1:
        raise ValueError("fewer samples than one mini-batch")
    rng = np.random.default_rng(seed)
    losses = np.zeros(epochs)
    for ep in range(epochs):
        perm = rng.permutation(samples)
        total = 0.0
        for s in range(steps):
            idx = perm[s * batch + rank * per: s * batch + (rank + 1) * per]
            g, loss = grad_fn(x[idx], t[idx])
            vec = np.concatenate([np.asarray(g, dtype=np.float32).ravel(),
                                  np.asarray([loss], dtype=np.float32)])
            vec = allreduce_mean(vec, world, device)
            step_fn(vec[:-1])
            total += float(vec[-1])
        losses[ep] = total / steps
    return losses
