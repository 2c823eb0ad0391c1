"""The split of one batch, and of the warm-start network's training, across
ranks (sovereign-solver_b200/shard.py), on the CPU: the partitioner's balance
and coverage, and two ranks over gloo on 127.0.0.1 -- the ordered gather of a
sharded batch (stand-in results) and data-parallel training (a stand-in model
whose gradients numpy computes) against the same training on one rank.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def shard(pkg):
    return pkg.shard


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_every_instance_once_and_balances_nonzeros(shard, world):
    rng = np.random.default_rng(world)
    w = rng.lognormal(8, 1.5, 500).astype(int) + 1
    parts = shard.partition(w, world)
    assert len(parts) == world
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(w)))
    for p in parts:
        assert p == sorted(p)
    loads = [w[p].sum() for p in parts]
    # greedy largest-first: no part exceeds another by more than the largest weight
    assert max(loads) - min(loads) <= w.max()
    assert shard.partition(w, world) == parts  # deterministic


def test_partition_edge_cases(shard):
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5, 5], 4) == [[0], [1], [], []]
    assert shard.partition([0, 0, 0], 2) == [[0, 2], [1]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def linear_model_grad(W, x, t):
    """Gradient of mean((x W^T - t)^2) over the rows and outputs."""
    r = x @ W.T - t
    return (2.0 / r.size) * (r.T @ x), float(np.mean(r * r))


def numpy_adam():
    state = {"m": None, "v": None, "t": 0}

    def step(W, g, lr=1e-2, b1=0.9, b2=0.999, eps=1e-8):
        if state["m"] is None:
            state["m"], state["v"] = np.zeros_like(g), np.zeros_like(g)
        state["t"] += 1
        state["m"] = b1 * state["m"] + (1 - b1) * g
        state["v"] = b2 * state["v"] + (1 - b2) * g * g
        c1, c2 = 1 - b1 ** state["t"], 1 - b2 ** state["t"]
        W -= lr * (state["m"] / c1) / (np.sqrt(state["v"] / c2) + eps)
    return step


def train(shard, rank, world, x, t):
    W = np.zeros((t.shape[1], x.shape[1]), dtype=np.float32)
    adam = numpy_adam()

    def grad_fn(xs, ts):
        g, loss = linear_model_grad(W, xs, ts)
        return g.astype(np.float32), loss

    def step_fn(g):
        adam(W, g.reshape(W.shape))

    losses = shard.train_data_parallel(x, t, epochs=5, batch=32, grad_fn=grad_fn, step_fn=step_fn,
                                       rank=rank, world=world, seed=7)
    return W, losses


def data():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((256, 6)).astype(np.float32)
    t = (x @ rng.standard_normal((6, 3)) + 0.1 * rng.standard_normal((256, 3))).astype(np.float32)
    return x, t


WORKER = textwrap.dedent("""
    import datetime, importlib, json, os, sys
    sys.path.insert(0, {root!r}); sys.path.insert(0, os.path.join({root!r}, "tests"))
    import numpy as np
    import torch.distributed as dist
    import test_shard_cpu as T
    pkg = importlib.import_module("sovereign-solver_b200")
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    out = {{"rank": rank}}
    # a sharded batch: stand-in problems, stand-in solves tagged with the rank
    class P:
        def __init__(self, k, nnz):
            self.k, self.nnz = k, nnz
    probs = [P(k, int(nnz)) for k, nnz in enumerate(np.random.default_rng(1).integers(1, 1000, 37))]
    res = pkg.shard.solve_sharded(probs, lambda ps: [{{"k": p.k, "rank": rank}} for p in ps],
                                  rank, world)
    out["gathered"] = res
    x, t = T.data()
    W, losses = T.train(pkg.shard, rank, world, x, t)
    out["W"] = W.tolist()
    out["losses"] = losses.tolist()
    dist.destroy_process_group()
    print("RESULT " + json.dumps(out))
""")


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gather_in_order_and_train_like_one(shard):
    code = WORKER.format(root=ROOT)
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        so, se = p.communicate(timeout=300)
        assert p.returncode == 0, se[-3000:]
        line = next(ln for ln in so.splitlines() if ln.startswith("RESULT "))
        outs.append(json.loads(line[len("RESULT "):]))
    r0, r1 = sorted(outs, key=lambda o: o["rank"])
    # rank 0 holds every result in instance order; the work was split
    assert r1["gathered"] is None
    assert [g["k"] for g in r0["gathered"]] == list(range(37))
    ranks = {g["rank"] for g in r0["gathered"]}
    assert ranks == {0, 1}
    # the replicas stay identical, and equal training on one rank with the
    # whole mini-batch (float32 sums in another order: 1e-5)
    assert np.array_equal(np.array(r0["W"]), np.array(r1["W"]))
    x, t = data()
    W1, losses1 = train(shard, 0, 1, x, t)
    np.testing.assert_allclose(np.array(r0["W"]), W1, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(r0["losses"], losses1, rtol=1e-4)
    assert r0["losses"][-1] < r0["losses"][0]
