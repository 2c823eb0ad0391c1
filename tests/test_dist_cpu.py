"""The N > 1 path of bench.py on the CPU: two ranks over gloo on 127.0.0.1.

Per rank: the reductions the bench times with (max over ranks of the device
time, sum over ranks of the units) and its barrier; the replica workload (one
LP per rank, the same shape, its own seed: weak scaling with no data-path
collective); and the reference arm under two ranks -- rank 0 alone prints its
one JSON line (n_gpus = 2), rank 1 exits without work.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import argparse, contextlib, datetime, importlib, io, json, os, sys
    sys.path.insert(0, {root!r})
    import torch.distributed as dist
    import bench
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    out = {{"rank": rank}}
    out["max"] = bench.max_over_ranks(1.5 + rank, world)
    out["sum"] = bench.sum_over_ranks(1.5 + rank, world)
    bench.barrier(world)
    pkg = importlib.import_module("sovereign-solver_b200")
    p = bench.replica_problem(pkg, rank, 12, 30)
    out["shape"] = [p.m, p.n, p.nnz]
    out["c_sum"] = float(p.c.sum())
    args = argparse.Namespace(supplies=12, demands=30, ref_iters_per_step=2, warmup=3, steps=2)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args)
    out["ref_lines"] = buf.getvalue().strip().splitlines()
    bench.barrier(world)
    dist.destroy_process_group()
    print("RESULT " + json.dumps(out))
""")


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_reduce_replicate_and_run_the_reference_on_rank_zero():
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
    for o in (r0, r1):
        assert o["max"] == 2.5 and o["sum"] == 4.0
    assert r0["shape"] == r1["shape"] == [42, 360, 720]
    assert r0["c_sum"] != r1["c_sum"]  # each replica has its own seed
    assert r1["ref_lines"] == []
    assert len(r0["ref_lines"]) == 1
    line = json.loads(r0["ref_lines"][0])
    assert line["impl"] == "reference"
    if "unavailable" not in line:  # the compiled reference is present
        assert line["n_gpus"] == 2 and line["value"] > 0
        assert line["e2e"]["h2d_bytes_per_step"] == 0
        assert line["cpu_baseline"]["kind"] == "reference"
