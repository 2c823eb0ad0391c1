"""Benchmark: PDHG on the 10M-column transportation LP (one B200 per rank).

Workload: 2,000 supplies x 5,000 demands = 10,000,000 columns, 7,000 rows,
20,000,000 nonzeros (all 1.0), costs U[1,100], x >= 0; mixed precision (FP32
iterates and SpMVs, FP64 residual / restart checks); PDLP's relative KKT
(termination rule 2) with adaptive restarts on its measure. Beside it: the
same steps in all-FP64 arithmetic (`fp64`), one full solve of the LP to 1e-4
(`full_solve`), the batched engine on 4,096 LPs (`batch`), the precision study
on the badly scaled LP (`precision`) and the learned warm start (`warmstart`).

A step is one call of the engine's solve on that LP running
`--iters-per-step` PDHG iterations (default 2,000 = 50 check periods) from the
cold start, with the problem resident in HBM (`value`), or end to end through
the C-ABI from pinned host memory: problem upload + scaling + solve + result
download (`e2e`).

Metric unit: SpMV HBM GB/s = B_spmv x iterations / second, with B_spmv the
algorithmic bytes of one iteration's two SpMVs on FP32 values and int32
indices, 16 nnz + 12 (m + n) = 440.1 MB for this LP (the same constant for
every implementation, so the GB/s ratio between two arms is their
iterations/s ratio).

Multi-GPU: the single-LP path does not shard; `--gpus N` runs N independent
replicas (one LP per rank, seed offset by rank), weak scaling, and reports the
whole-job aggregate over the max-over-ranks device time.

`--impl reference` times the reference's own CPU PDHG (the reference PDHG
path compiled from its sources, oracle/_ref) on the same LP: one stock
Pdhg::solve call whose per-iteration timestamps (taken by a forwarding Backend
decorator, outside the algorithm) give the loop throughput.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LPs solved/s at 1e-4 rel KKT: learned+batched vs plain GPU PDHG; SpMV HBM GB/s"
UNIT = "GB/s"
SUPPLIES, DEMANDS = 2000, 5000


def workload_name(supplies: int, demands: int) -> str:
    """The LP both arms solve (the arithmetic is each arm's `dtype`)."""
    return (f"transportation LP {supplies:,} x {demands:,} ({supplies * demands:,} columns, "
            f"{supplies + demands:,} rows, {2 * supplies * demands:,} nnz), PDHG iterations")


def bench_config(args, world: int) -> dict:
    """The `config` object, identical in both arms' lines."""
    return {"workload": workload_name(args.supplies, args.demands),
            "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (resident set ~1.3 GB > 126 MB)"}


# Options of the solves: PDLP's relative KKT (termination rule 2), adaptive
# restarts on its measure and the reflected restarted Halpern iteration (on
# one B200: 13,200 instead of 29,160 iterations for the transportation LP,
# 1.4x the batch's solves/s). The primal weight stays 1 on the transportation
# LP: its update drives omega from |c|/|b| ~ 135 towards 0.1 there and costs
# 2-3x the iterations (oracle, 100 x 250 and 200 x 500 instances of the
# family); the other workloads turn it on.
HEADLINE = dict(termination_rule="relative_kkt_l2", restart_rule="adaptive_l2", halpern=True)


def replica_problem(pkg, rank: int, supplies: int = SUPPLIES, demands: int = DEMANDS):
    """The LP one replica solves: the same shape on every rank, its own seed."""
    return pkg.lpgen.transportation_lp(supplies, demands, seed=1000 + rank)


def spmv_bytes(m: int, n: int, nnz: int) -> float:
    return 16.0 * nnz + 12.0 * (m + n)


def load_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlClockSampler:
    """The same fields read in this process through NVML (a thread polling
    every 200 ms), without a second process querying the GPU. The device is
    found by its PCI bus id, so the index under CUDA_VISIBLE_DEVICES does not
    matter."""

    def __init__(self, device: int):
        self.device = device
        self.samples: list[tuple[float, float, int]] = []
        self.max_mhz = None
        self.handle = None
        self.nvml = None
        self.halt = threading.Event()
        self.thread = None

    def start(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            props = torch.cuda.get_device_properties(self.device)
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
        except Exception:
            self.handle = None
            return
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()

    def _poll(self):
        n = self.nvml
        while not self.halt.is_set():
            try:
                self.samples.append((n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM),
                                     n.nvmlDeviceGetPowerUsage(self.handle) / 1e3,
                                     n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)))
            except Exception:
                pass
            self.halt.wait(0.2)

    def stop(self) -> dict:
        if self.handle is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable"]}
        self.halt.set()
        self.thread.join(timeout=5)
        n = self.nvml
        bits = {"hw_slowdown": n.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": n.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": n.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": n.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted(k for k, b in bits.items() if any(s[2] & b for s in self.samples))
        sm = [s[0] for s in self.samples]
        try:
            n.nvmlShutdown()
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(sm), "source": "nvml"}


def parse_cpulist(text: str) -> set[int]:
    """"0-3,8,10-11" (the sysfs cpulist format) -> {0, 1, 2, 3, 8, 10, 11}."""
    out: set[int] = set()
    for part in text.strip().split(","):
        part = part.strip()
        if not part:
            continue
        if "-" in part:
            a, b = part.split("-")
            out.update(range(int(a), int(b) + 1))
        else:
            out.add(int(part))
    return out


class NearGpu:
    """Binds this process to the host cores of the GPU's own NUMA node (sysfs
    local_cpulist of its PCI function) while the e2e steps allocate their
    pinned buffers and run, then restores the previous affinity: pinned pages
    are placed on the node of the thread that first touches them, and DMA from
    the other socket's memory crosses the inter-socket link. Without sysfs or
    with no overlap with the allowed cores it changes nothing."""

    def __init__(self, device: int, sysfs: str = "/sys/bus/pci/devices"):
        self.device = device
        self.sysfs = sysfs
        self.saved = None
        self.cpus: set[int] = set()
        self.bound = False

    def local_cpus(self) -> set[int]:
        import torch
        p = torch.cuda.get_device_properties(self.device)
        bus = f"{p.pci_domain_id:04x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        with open(os.path.join(self.sysfs, bus, "local_cpulist")) as f:
            return parse_cpulist(f.read())

    def __enter__(self) -> "NearGpu":
        try:
            allowed = os.sched_getaffinity(0)
            cpus = self.local_cpus() & allowed
            if cpus and cpus != allowed:
                self.saved = allowed
                os.sched_setaffinity(0, cpus)
                self.bound = True
            self.cpus = cpus
        except Exception:
            self.cpus = set()
        return self

    def __exit__(self, *exc) -> None:
        if self.saved is not None:
            os.sched_setaffinity(0, self.saved)
            self.saved = None

    def describe(self) -> str:
        if not self.cpus:
            return "pinned; the GPU's NUMA node unknown, affinity unchanged"
        if not self.bound:
            return f"pinned; every allowed core ({len(self.cpus)}) is local to the GPU"
        return f"pinned, allocated and driven from the GPU's NUMA node ({len(self.cpus)} cores)"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _reduce(v: float, op: str) -> float:
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(v: float, world: int) -> float:
    """The largest v of all ranks (the job's time is its slowest rank's)."""
    return v if world == 1 else _reduce(v, "max")


def sum_over_ranks(v: float, world: int) -> float:
    """The sum of v over all ranks (whole-job units)."""
    return v if world == 1 else _reduce(v, "sum")


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def traffic_from_profile() -> float | None:
    """DRAM bytes per launch of the primal kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "primal_transportation_10M.json")
    try:
        with open(path) as f:
            return float(json.load(f)["dram_bytes_per_launch"])
    except Exception:
        return None


def cpu_baseline_port(prob, iters: int = 12) -> dict:
    """The oracle's C restatement, 1 core, a bounded sample: `iters` iterations after setup."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    t = np.zeros(iters)
    t0 = time.perf_counter()
    orc.oracle_solve(prob, max_iterations=iters, iter_times=t, tolerance=1e-12)
    wall = time.perf_counter() - t0
    per_it = float(np.mean(np.diff(t)))
    b = spmv_bytes(prob.m, prob.n, prob.nnz)
    return {"value": b / per_it / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{iters} PDHG iterations of the same LP after setup "
                      f"({per_it * 1e3:.1f} ms/iteration; whole call incl. setup {wall:.1f} s)",
            "iterations_per_s": 1.0 / per_it}


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    if not orc.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libsovref.so not built (needs the reference sources)"}))
        return
    pkg = importlib.import_module("sovereign-solver_b200")
    prob = replica_problem(pkg, 0, args.supplies, args.demands)
    per_step = args.ref_iters_per_step
    total = (args.warmup + args.steps) * per_step + 1
    t = np.zeros(total)
    t0 = time.perf_counter()
    r = orc.reference_solve(prob, max_iterations=total, iter_times=t, tolerance=1e-12)
    wall = time.perf_counter() - t0
    starts = t[args.warmup * per_step: total: per_step]
    step_s = np.diff(starts)
    ms = float(np.mean(step_s)) * 1e3
    b = spmv_bytes(prob.m, prob.n, prob.nnz)
    value = b * per_step / (ms / 1e3) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded transportation LP)",
        "config": bench_config(args, world),
        "iterations_per_step": per_step,
        "implementation": "reference sov::Pdhg::solve, Host backend (single-threaded), FP64",
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"{args.steps} steps x {per_step} iterations of one stock "
                                   f"Pdhg::solve call after {args.warmup} warm-up steps; whole "
                                   f"call incl. the reference's setup {wall:.1f} s"},
        "iterations_per_s": per_step / (ms / 1e3),
        "reference_status": r.status,
    }
    print(json.dumps(line))


def batch_line(pkg, eng, args, rank: int, world: int = 1) -> dict:
    """Config 3: a seeded family of config-0-structure LPs (m log-uniform in
    [50, 5000], n = 2-3 m, 4-10 nonzeros per column), solved to 1e-4 relative
    KKT by the batched engine (pdhg_solve_batch: one CUDA-graph launch per
    rank), beside the plain single-LP engine on an evenly spaced sample of the
    same family. With N ranks the family has N x --batch-instances LPs and
    shard.solve_sharded splits it by balanced nonzeros, one batched solve per
    rank, results gathered to rank 0 in instance order (weak scaling; no
    per-iteration collective)."""
    ps = pkg.lpgen.batch_family(args.batch_instances * world, seed_base=3000)
    opt = pkg.PdhgOptions(precision="mixed", tolerance=1e-4, max_iterations=200_000,
                          primal_weight_update=True, **HEADLINE)
    # the plain engine solves an evenly spaced sample of the same instances
    step = max(1, len(ps) // max(1, args.plain_instances))
    sample = list(range(0, len(ps), step))[: args.plain_instances]
    loads = []
    with pkg.Engine(eng.device) as e:
        e.load_batch(ps[: min(len(ps), 64)])
        e.solve_batch(opt, want_point=False)  # warm-up (graph build, clocks)

        def solve_part(part):
            t = time.perf_counter()
            e.load_batch(part)
            loads.append(time.perf_counter() - t)
            return e.solve_batch(opt, want_point=False)

        barrier(world)
        t0 = time.perf_counter()
        rs = pkg.shard.solve_sharded(ps, solve_part, rank, world)
        t_batch = max_over_ranks(time.perf_counter() - t0, world)
        t_load = max_over_ranks(loads[0] if loads else 0.0, world)
        plain, t_plain = [], 1.0
        if rank == 0:
            t0 = time.perf_counter()
            for k in sample:
                e.load(ps[k])
                plain.append(e.solve(opt, want_point=False))
            t_plain = time.perf_counter() - t0
    if rank != 0:
        return {}
    solved = sum(r.status == "optimal" for r in rs)
    plain_solved = sum(r.status == "optimal" for r in plain)
    its = sorted(r.iterations for r in rs)
    fp64_its = sum(r.fp64_iterations for r in rs)
    return {"workload": f"{len(ps)} seeded LPs, m log-uniform [50, 5000], n = 2-3 m, "
                        f"4-10 nnz/column ({sum(p.nnz for p in ps):,} nnz), PDLP relative KKT "
                        f"1e-4, mixed, adaptive restarts, Halpern iteration, primal weight",
            "instances": len(ps), "ranks": world, "solved": solved, "seconds": t_batch,
            "load_seconds": t_load, "solves_per_s": solved / t_batch,
            "solves_per_s_problem_resident": solved / max(t_batch - t_load, 1e-9),
            "iterations_median": its[len(its) // 2], "iterations_max": its[-1],
            "polished": sum(r.fp64_iterations > 0 for r in rs),
            "fp64_iteration_fraction": fp64_its / max(1, sum(its)),
            "gpu_launches": rs[0].kernel_launches if rs else 0,
            "plain_gpu": {"instances": len(plain), "sample": f"every {step}th instance of the "
                          f"same family ({len(plain)} of {len(ps)}), on rank 0",
                          "solved": plain_solved,
                          "seconds": t_plain, "solves_per_s": plain_solved / t_plain},
            "speedup_vs_plain_gpu": (solved / t_batch) / (plain_solved / t_plain)
            if plain_solved else None,
            "timing": "host wall clock around load + solve (pdhg_load_batch + pdhg_solve_batch "
                      "per rank, the gather to rank 0 included, max over ranks); the plain "
                      "engine per instance pdhg_load_problem + pdhg_solve"}


def precision_line(pkg, eng, args, rank: int) -> dict:
    """Config 2: the badly scaled LP (200,000 rows, 500,000 columns, 8
    nonzeros per column at power-law rows, magnitudes log-uniform in
    [1e-3, 1e3], 30% <= rows, boxes), solved from the cold start under the
    same iteration budget and 1e-4 relative-KKT rule by the all-FP64 mode, the
    FP32-bulk / FP64-check mode (FP64 polish once the FP32 phase stalls) and
    the same without the polish (FP32 iterates to the end). Each arm's
    objective error is taken against the FP64 run."""
    p = pkg.lpgen.badly_scaled_lp(200_000, 500_000, 8, seed=2000 + rank)
    out = {"workload": f"badly scaled LP {p.m:,} x {p.n:,}, {p.nnz:,} nnz (power-law rows, "
                       f"|a| log-uniform [1e-3, 1e3], 30% <= rows), PDLP relative KKT 1e-4, "
                       f"adaptive restarts, Halpern iteration, primal weight",
           "iteration_budget": args.precision_iters}
    arms = {"fp64": dict(precision="fp64"), "mixed": dict(precision="mixed"),
            "fp32_only": dict(precision="mixed", polish_iterations=0)}
    with pkg.Engine(eng.device) as e:
        e.load(p)
        for name, kw in arms.items():
            o = pkg.PdhgOptions(primal_weight_update=True, tolerance=1e-4,
                                max_iterations=args.precision_iters, **HEADLINE, **kw)
            r = e.solve(o, want_point=False)
            out[name] = {"status": r.status, "iterations": r.iterations,
                         "relative_kkt": r.relative_kkt, "objective": r.objective,
                         "fp64_iterations": r.fp64_iterations,
                         "fp64_iteration_fraction": r.fp64_iterations / max(1, r.iterations),
                         "device_seconds": r.device_seconds,
                         "iterations_per_s": r.iterations / r.device_seconds
                         if r.device_seconds > 0 else None,
                         "b_spmv_gb_per_s": spmv_bytes(p.m, p.n, p.nnz) * r.iterations
                         / r.device_seconds / 1e9 if r.device_seconds > 0 else None}
        out["tuning"] = {"fp64": e.tuning("fp64"), "mixed": e.tuning("mixed")}
    ref = out["fp64"]["objective"]
    out["fp64_reference"] = ("the all-FP64 arm's objective" if out["fp64"]["status"] == "optimal"
                             else "the all-FP64 arm did not converge: errors compare "
                                  "unconverged points")
    for name in ("mixed", "fp32_only"):
        out[name]["objective_error_vs_fp64"] = (abs(out[name]["objective"] - ref)
                                                / max(1.0, abs(ref)))
    return out


def warmstart_line(pkg, eng, args, rank: int) -> dict:
    """Config 4 at reduced size: a parametric family over a config-2-structure
    base (500 rows, 1,200 columns, 6,000 nonzeros; 64 parameters moving b and
    c by ~10%). Training solves from the batched engine, basis + network
    (tensor-core training), then on held-out parameters: plain single-LP GPU
    PDHG from the cold start, batched cold, and batched with the gated learned
    warm start and the cold fallback past the family's iteration budget.
    Solves/s include, for the warm line, prediction, gating and the fallback's
    cold solves."""
    W = pkg.warmstart
    fam = pkg.lpgen.parametric_family(500, 1200, 5, seed=4001)
    opt = pkg.PdhgOptions(precision="mixed", primal_weight_update=True, tolerance=1e-4,
                          max_iterations=300_000, **HEADLINE)
    tr_th = fam.thetas(args.ws_train, seed=1 + 1000 * rank)
    te_th = fam.thetas(args.ws_test, seed=2 + 1000 * rank)
    tr = [fam.instance(t) for t in tr_th]
    te = [fam.instance(t) for t in te_th]
    with pkg.Engine(eng.device) as e:
        t0 = time.perf_counter()
        res = W.solve_family(e, tr, opt)
        t_train_solves = time.perf_counter() - t0
        ws = W.LearnedWarmStart(fam, rank=64, hidden=512, device=eng.device)
        t0 = time.perf_counter()
        rep = ws.fit(tr_th, res, epochs=600, batch=64, lr=1e-3)
        t_fit = time.perf_counter() - t0
        W.solve_family(e, te[:8], opt)  # warm-up
        t0 = time.perf_counter()
        cold = W.solve_family(e, te, opt)
        t_cold = time.perf_counter() - t0
        t0 = time.perf_counter()
        x0s, y0s, used, kw, kc = ws.starts(e, te, te_th, opt)
        warm = W.solve_family_with_fallback(e, te, opt, x0s, y0s, ws.budget)
        t_warm = time.perf_counter() - t0
        t0 = time.perf_counter()
        plain = []
        for p in te[: args.plain_instances]:
            e.load(p)
            plain.append(e.solve(opt, want_point=False))
        t_plain = time.perf_counter() - t0
    ok = lambda rs: sum(r.status == "optimal" for r in rs)  # noqa: E731
    plain_rate = ok(plain) / t_plain
    warm_rate = ok(warm) / t_warm
    it_c = np.array([r.iterations for r in cold], dtype=float)
    it_w = np.array([r.iterations for r in warm], dtype=float)
    ratio = it_w / np.maximum(it_c, 1.0)  # per held-out instance, warm over cold
    cap = opt.max_iterations
    return {"workload": f"parametric family over a config-2-structure base (500 x 1,200, 6,000 "
                        f"nnz, 64 parameters, b and c moved ~10%); {len(tr)} training solves, "
                        f"{len(te)} held-out; mixed, PDLP relative KKT 1e-4, adaptive restarts, "
                        f"Halpern iteration, primal weight",
            "training": {"solves_s": t_train_solves, "solved": ok(res), "fit_s": t_fit,
                         "basis_rank": rep.rank, "explained_primal": rep.explained_primal,
                         "explained_dual": rep.explained_dual, "val_loss": ws.val_loss},
            "gate": {"warm_used": int(used.sum()), "start_kkt_warm_median": float(np.median(kw)),
                     "start_kkt_cold_median": float(np.median(kc))},
            "plain_gpu": {"instances": len(plain),
                          "sample": f"the first {len(plain)} of the {len(te)} held-out instances "
                                    f"(the batched arms solve all {len(te)})",
                          "solved": ok(plain), "seconds": t_plain, "solves_per_s": plain_rate,
                          "iterations_mean": float(np.mean([r.iterations for r in plain])),
                          "batched_cold_iterations_mean_same_sample":
                              float(np.mean(it_c[: len(plain)]))},
            "batched_cold": {"solved": ok(cold), "seconds": t_cold, "solves_per_s": ok(cold) / t_cold,
                             "iterations_mean": float(it_c.mean()),
                             "iterations_median": float(np.median(it_c)),
                             "iterations_max": int(it_c.max()), "at_cap": int((it_c >= cap).sum())},
            "batched_learned_warm": {"solved": ok(warm), "seconds": t_warm,
                                     "solves_per_s": warm_rate,
                                     "iterations_mean": float(it_w.mean()),
                                     "iterations_median": float(np.median(it_w)),
                                     "iterations_max": int(it_w.max()),
                                     "at_cap": int((it_w >= cap).sum()),
                                     "fallback": {"budget": int(ws.budget),
                                                  "solved_again_cold": int((it_w > ws.budget).sum()),
                                                  "rule": "a warm solve gets the most iterations "
                                                          "any training solve needed; one not "
                                                          "optimal by then is solved again from "
                                                          "the cold start (iterations of both "
                                                          "attempts counted)"},
                                     "max_relative_kkt": float(max(r.relative_kkt for r in warm
                                                                   if r.status == "optimal"))},
            "warm_over_cold_iterations": {"median": float(np.median(ratio)),
                                          "geometric_mean": float(np.exp(np.mean(np.log(
                                              np.maximum(ratio, 1e-9))))),
                                          "instances_faster": int((ratio < 1.0).sum()),
                                          "instances": int(ratio.size)},
            "speedup_vs_plain_gpu": warm_rate / plain_rate if plain_rate > 0 else None,
            "timing": "host wall clock; batched lines include load, the warm line also "
                      "prediction and the start-KKT gate"}


def profile_case(args) -> None:
    """The ncu target: one mixed-precision solve of --iters-per-step iterations
    (FP32 to the end, no polish). --profile-lp transportation: the
    transportation LP of --supplies x --demands; badly_scaled: the 200,000 x
    500,000 badly scaled LP; batch: the first --batch-instances LPs of the
    batched family in one batched solve (below one check period, 40
    iterations, the iteration kernels launch one by one instead of inside the
    solve graph); mlp: --iters-per-step Adam steps of the warm start's network
    (64 -> 512 -> 512 -> 512, mini-batches of 256) on random data."""
    import torch
    torch.cuda.set_device(0)
    pkg = importlib.import_module("sovereign-solver_b200")
    opt = dict(precision="mixed", tolerance=1e-12, polish_iterations=0,
               max_iterations=args.iters_per_step, **HEADLINE)
    if args.profile_lp == "mlp":
        rng = np.random.default_rng(0)
        x = rng.standard_normal((4096, 64)).astype(np.float32)
        t = rng.standard_normal((4096, 512)).astype(np.float32)
        with pkg.mlp.Mlp(64, 512, 512, max_batch=256) as net:
            steps = max(1, args.iters_per_step)
            net.train(x[: 256 * steps], t[: 256 * steps], epochs=1, batch=256)
        print(json.dumps({"profile_case": "mlp 64-512-512-512", "adam_steps": steps}))
        return
    if args.profile_lp == "batch":
        ps = pkg.lpgen.batch_family(args.batch_instances, seed_base=3000)
        with pkg.Engine(0) as eng:
            eng.load_batch(ps)
            rs = eng.solve_batch(pkg.PdhgOptions(primal_weight_update=True, **opt),
                                 want_point=False)
            tuning = eng.batch_tuning("mixed")
        print(json.dumps({"profile_case": f"batch of {len(ps)} LPs ({sum(p.nnz for p in ps)} nnz)",
                          "iterations": max(r.iterations for r in rs), "tuning": tuning}))
        return
    if args.profile_lp == "badly_scaled":
        prob = pkg.lpgen.badly_scaled_lp(200_000, 500_000, 8, seed=2000)
        name = "badly scaled 200000x500000"
        opt["primal_weight_update"] = True
    else:
        prob = pkg.lpgen.transportation_lp(args.supplies, args.demands, seed=1000)
        name = f"transportation {args.supplies}x{args.demands}"
    with pkg.Engine(0) as eng:
        eng.load(prob)
        # a first short solve runs the autotuner and captures the period's
        # graph; the measured solve sits in the NVTX range "measured" (ncu
        # --nvtx --nvtx-include "measured/" keeps the tuner's launches out)
        eng.solve(pkg.PdhgOptions(**dict(opt, max_iterations=40)), want_point=False)
        torch.cuda.nvtx.range_push("measured")
        r = eng.solve(pkg.PdhgOptions(**opt), want_point=False)
        torch.cuda.nvtx.range_pop()
        tuning = eng.tuning("mixed")
    print(json.dumps({"profile_case": name, "iterations": r.iterations, "status": r.status,
                      "tuning": tuning}))


def mps_reader_line(args) -> None:
    """Read throughput of the MPS reader (host threads, no device): the
    transportation LP of --supplies x --demands written as MPS text, read by
    pdhg_read_mps with all host threads and with one; the reference's
    read_mps_string (oracle/_ref, one thread, as it is written) on the same
    model at --mps-ref-supplies supplies. Bytes of text per second."""
    import ctypes as C
    pkg = importlib.import_module("sovereign-solver_b200")
    L = pkg.mps._lib()

    def text_of(supplies):
        p = pkg.lpgen.transportation_lp(supplies, args.demands, seed=1000)
        return pkg.mps.write_mps(p).encode(), p

    def ours(text, threads):
        o = pkg.mps._MpsOptions(0, 1, threads)
        h, err = C.c_void_p(), C.create_string_buffer(4096)
        t = time.perf_counter()
        rc = L.pdhg_read_mps(text, len(text), None, C.byref(o), C.byref(h), err, len(err))
        dt = time.perf_counter() - t
        if rc != 0:
            raise RuntimeError(err.value.decode())
        L.pdhg_model_free(h)
        return dt

    text, p = text_of(args.supplies)
    cores = os.cpu_count() or 1
    all_t = min(ours(text, 0) for _ in range(3))
    one_t = ours(text, 1)
    line = {"metric": "mps_read_throughput", "value": round(len(text) / all_t / 1e6, 1),
            "unit": "MB/s", "higher_is_better": True, "threads": cores,
            "seconds": round(all_t, 3), "single_thread_MBps": round(len(text) / one_t / 1e6, 1),
            "config": {"workload": f"transportation {args.supplies}x{args.demands} as MPS text",
                       "bytes": len(text), "rows": p.m, "columns": p.n, "nonzeros": p.nnz},
            "data": "synthetic"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc  # the reference reader, where oracle/_ref is built
    if orc.ref_available() and args.mps_ref_supplies > 0:
        rtext, rp = text_of(args.mps_ref_supplies)
        R = orc.ref_lib()
        orc.reference_read_mps("ROWS\n N c\n")  # declares the entry points
        err = C.create_string_buffer(4096)
        t = time.perf_counter()
        h = R.ref_read_mps(rtext, len(rtext), b"<string>", 0, 1, err, len(err))
        rt = time.perf_counter() - t
        R.ref_model_free(h)
        ours_same = min(ours(rtext, 0) for _ in range(3))
        line["reference"] = {"value": round(len(rtext) / rt / 1e6, 1), "unit": "MB/s", "cores": 1,
                             "kind": "reference", "seconds": round(rt, 3),
                             "sample": f"transportation {args.mps_ref_supplies}x{args.demands} "
                                       f"({len(rtext)} bytes, {rp.nnz} nonzeros)",
                             "ours_on_the_sample_MBps": round(len(rtext) / ours_same / 1e6, 1)}
    else:
        line["reference"] = {"unavailable": "oracle/_ref not built"}
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--iters-per-step", type=int, default=2000)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--ref-iters-per-step", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--full-solve-cap", type=int, default=100_000)
    ap.add_argument("--fp64-steps", type=int, default=3,
                    help="steps of the same LP in all-FP64 arithmetic (0 = skip)")
    ap.add_argument("--batch-instances", type=int, default=4096,
                    help="config-3 family size for the batched line (0 = skip)")
    ap.add_argument("--plain-instances", type=int, default=32,
                    help="an evenly spaced sample of that family solved one at a time")
    ap.add_argument("--ws-train", type=int, default=1024,
                    help="config-4 training solves for the learned warm start (0 = skip)")
    ap.add_argument("--ws-test", type=int, default=128, help="config-4 held-out instances")
    ap.add_argument("--precision-iters", type=int, default=100_000,
                    help="iteration budget per mode of the config-2 precision study (0 = skip)")
    ap.add_argument("--profile-lp", default="transportation",
                    choices=["transportation", "badly_scaled", "batch", "mlp"],
                    help="the LP of --profile-case")
    ap.add_argument("--profile-case", action="store_true",
                    help="profiler target: load the LP and run one solve of --iters-per-step "
                         "iterations, nothing else")
    ap.add_argument("--supplies", type=int, default=SUPPLIES)
    ap.add_argument("--demands", type=int, default=DEMANDS)
    ap.add_argument("--clock-sampler", default="nvidia-smi", choices=["nvidia-smi", "nvml"],
                    help="how clocks are sampled during the timed region: an nvidia-smi "
                         "process (-lms 200) or NVML read in this process every 200 ms")
    ap.add_argument("--mps-reader", action="store_true",
                    help="measure the MPS reader instead (host only, one JSON line)")
    ap.add_argument("--mps-ref-supplies", type=int, default=200,
                    help="supplies of the model the reference's reader is timed on")
    args = ap.parse_args()
    if args.mps_reader:
        mps_reader_line(args)
        return
    if args.profile_case:
        profile_case(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    pkg = importlib.import_module("sovereign-solver_b200")
    prob = replica_problem(pkg, rank)
    m, n, nnz = prob.m, prob.n, prob.nnz
    b_spmv = spmv_bytes(m, n, nnz)
    eng = pkg.Engine(local)
    eng.load(prob)
    opts = pkg.PdhgOptions(precision="mixed", tolerance=1e-12, max_iterations=args.iters_per_step,
                           **HEADLINE)
    stream = torch.cuda.ExternalStream(eng.stream_handle())

    # ---- device-resident throughput (value) ----
    for _ in range(args.warmup):
        eng.solve(opts, want_point=False)
    torch.cuda.synchronize()
    barrier(world)
    sampler = (NvmlClockSampler if args.clock_sampler == "nvml" else ClockSampler)(local)
    sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    barrier(world)
    ev0.record(stream)
    its = 0
    launches = 0
    for _ in range(args.steps):
        r = eng.solve(opts, want_point=False)
        its += r.iterations
        launches += r.kernel_launches
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    t_local = ev0.elapsed_time(ev1) / 1e3
    t_max = max_over_ranks(t_local, world)
    total_units = sum_over_ranks(b_spmv * its, world)
    value = total_units / t_max / 1e9
    ms_per_step = t_max * 1e3 / args.steps

    # ---- roofline of the dominant kernel (CUDA events on the engine's stream) ----
    peaks = load_peaks()
    ks = eng.profile_kernels("mixed", warmup=5, iterations=50)
    dom = max(ks[:2], key=lambda k: k["avg_ms"])
    achieved = dom["bytes"] / (dom["avg_ms"] / 1e3) / 1e9
    # the same pass by the generic per-row formula (row pointer and bounds
    # loaded, every index loaded): the lean Halpern primal touches six
    # vectors per column, two more once a check period
    rows, cols = (n, m) if dom["name"] == "primal" else (m, n)
    touches = (6 + 2 / 40) if dom["name"] == "primal" else (8 + 1 / 40)
    generic = 4 * (rows + 1) + 8 * nnz + 4 * cols + 4 * touches * rows
    roofline = {"bound": "hbm", "kernel": dom["name"], "achieved": achieved,
                "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                "peak_source": peaks["source"], "traffic": traffic_from_profile(),
                "algorithmic_bytes_per_launch": dom["bytes"],
                "bytes_note": "this LP's: the row pointer (every column has 2 entries) and the "
                              "column bounds (all 0 <= x) carry no information and are not loaded",
                "generic_bytes_per_launch": generic, "avg_launch_ms": dom["avg_ms"],
                "kernels": ks, "tuning": eng.tuning("mixed")}

    # ---- end to end through the C-ABI from pinned host memory (e2e) ----
    near = NearGpu(local).__enter__()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h = {k: pin(getattr(prob, k)) for k in ("row_ptr", "col_idx", "val", "c", "col_lo",
                                               "col_hi", "row_lo", "row_hi")}
    out_x = torch.empty(n, dtype=torch.float64).pin_memory()
    out_y = torch.empty(m, dtype=torch.float64).pin_memory()
    out_rc = torch.empty(n, dtype=torch.float64).pin_memory()
    lib = pkg.pdhg.lib()
    import ctypes as C
    dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))  # noqa: E731
    ip = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_int32))  # noqa: E731
    eng2 = pkg.Engine(local)
    o = pkg.pdhg._Options()
    lib.pdhg_default_options(C.byref(o))
    o.precision, o.tolerance = 1, 1e-12
    o.termination_rule = pkg.pdhg.TERMINATION_RULES[HEADLINE["termination_rule"]]
    o.restart_rule = pkg.pdhg.RESTART_RULES[HEADLINE["restart_rule"]]
    o.halpern = 1 if HEADLINE["halpern"] else 0
    o.max_iterations = args.iters_per_step
    info = pkg.pdhg._Info()

    def e2e_step():
        rc = lib.pdhg_load_problem(eng2._h, m, n, nnz, ip(h["row_ptr"]), ip(h["col_idx"]),
                                   dp(h["val"]), dp(h["c"]), 0.0, 0, dp(h["col_lo"]),
                                   dp(h["col_hi"]), dp(h["row_lo"]), dp(h["row_hi"]))
        assert rc == 0, lib.pdhg_last_error(eng2._h)
        rc = lib.pdhg_solve(eng2._h, C.byref(o), C.byref(info), dp(out_x), dp(out_y), dp(out_rc))
        assert rc == 0, lib.pdhg_last_error(eng2._h)
        return info.iterations

    e2e_step()  # warm-up
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    e_its = 0
    for _ in range(args.e2e_steps):
        e_its += e2e_step()
    torch.cuda.synchronize()
    e_t = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = sum_over_ranks(b_spmv * e_its, world) / e_t / 1e9
    h2d = sum(int(t.numel() * t.element_size()) for t in h.values())
    d2h = int((2 * n + m) * 8)
    eng2.close()
    near.__exit__(None, None, None)

    # ---- the same steps in all-FP64 arithmetic (same-precision comparison
    # with the FP64 reference arm) ----
    fp64 = None
    if args.fp64_steps > 0:
        o64 = pkg.PdhgOptions(precision="fp64", tolerance=1e-12,
                              max_iterations=args.iters_per_step, **HEADLINE)
        eng.solve(o64, want_point=False)  # warm-up (and the FP64 shapes' tuning)
        f_its, f_t = 0, 0.0
        for _ in range(args.fp64_steps):
            r = eng.solve(o64, want_point=False)
            f_its += r.iterations
            f_t += r.device_seconds
        f_t = max_over_ranks(f_t, world)
        fp64 = {"value": sum_over_ranks(b_spmv * f_its, world) / f_t / 1e9, "unit": UNIT,
                "iterations_per_s": sum_over_ranks(f_its, world) / f_t, "steps": args.fp64_steps,
                "dtype": "f64", "tuning": eng.tuning("fp64"),
                "timing": "CUDA events around each solve's iteration loop (device_seconds), "
                          "problem resident in HBM"}

    # ---- one full solve to 1e-4 relative KKT (LPs solved/s, reported beside) ----
    solve_opts = pkg.PdhgOptions(precision="mixed", tolerance=1e-4,
                                 max_iterations=args.full_solve_cap, **HEADLINE)
    t0 = time.perf_counter()
    full = eng.solve(solve_opts, want_point=False)
    full_s = time.perf_counter() - t0

    batch = batch_line(pkg, eng, args, rank, world) if args.batch_instances > 0 else None
    warm = warmstart_line(pkg, eng, args, rank) if args.ws_train > 0 else None
    prec = precision_line(pkg, eng, args, rank) if args.precision_iters > 0 else None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded transportation LP, one per rank)",
        "config": bench_config(args, world),
        "iterations_per_step": args.iters_per_step,
        "b_spmv_bytes_per_iteration": b_spmv,
        "options": "FP32 iterates, FP64 checks; PDLP relative KKT (rule 2), adaptive restarts "
                   "on its measure, reflected Halpern iteration, primal weight 1; tolerance "
                   "1e-12 in the timed steps (fixed work per step)",
        "iterations_per_s": sum_over_ranks(its, world) / t_max,
        "clocks": clocks,
        "gpu_launches": launches,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
                "ms_per_step": e_t * 1e3 / args.e2e_steps, "host_buffers": near.describe()},
        "roofline": roofline,
        "full_solve": {"status": full.status, "iterations": full.iterations,
                       "relative_kkt": full.relative_kkt, "seconds": full_s,
                       "device_seconds": full.device_seconds,
                       "lps_solved_per_s": (1.0 / full_s) if full.status == "optimal" else 0.0,
                       "restarts": full.restarts, "objective": full.objective,
                       "fp64_iterations": full.fp64_iterations,
                       "measure": "PDLP relative KKT (termination rule 2) < 1e-4, mixed, "
                                  "problem resident; host wall clock around pdhg_solve"},
    }
    if fp64 is not None:
        line["fp64"] = fp64
    if batch is not None:
        line["batch"] = batch
    if warm is not None:
        line["warmstart"] = warm
    if prec is not None:
        line["precision"] = prec
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(prob)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
