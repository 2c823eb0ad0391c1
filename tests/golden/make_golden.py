"""Regenerates the golden fixtures in this directory from the REFERENCE itself.

Run in a container that has the reference sources, after
``make -C oracle ref REF_SRC=<reference source tree>``:

    REF_SRC=<reference source tree> python tests/golden/make_golden.py [c0]

(`c0` regenerates only the two 2,000 x 5,000 fixtures.)

Every expected value stored here comes from the reference's own code: its LP
and MPS readers parse the models, its ``sov::Pdhg::solve`` on the Host backend
(oracle/_ref/libsovref.so, compiled from the reference sources) produces the
results, and its Host backend produces the SpMV answers. Inputs are taken from
the reference's own test and smoke files (tests/test_pdhg.cpp,
tests/test_l0_backend.cpp, tests/test_scaling.cpp, benchmarks/smoke/*.mps),
read as text here, plus seeded synthetic LPs from the engine's generators.
The GPU box has no reference sources; the tests there read only these files.
"""
from __future__ import annotations

import hashlib
import importlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import orc  # noqa: E402

pkg = importlib.import_module("sovereign-solver_b200")
REF_SRC = os.environ.get("REF_SRC", "")
if not os.path.isfile(os.path.join(REF_SRC, "src", "l1", "pdhg.cpp")):
    sys.exit("make_golden.py: set REF_SRC to the reference's source tree")

PROBLEM_KEYS = ("m", "n", "row_ptr", "col_idx", "val", "c", "col_lo", "col_hi", "row_lo",
                "row_hi", "obj_const", "maximize")


def _c_string_literals(body: str) -> str:
    """The LP text of a TEST body: a raw string R"(...)" or adjacent "..." literals."""
    raw = re.search(r'R"\((.*?)\)"', body, re.S)
    if raw:
        return raw.group(1)
    m = re.search(r'const char\* text\s*=\s*((?:"(?:[^"\\]|\\.)*"\s*)+);', body, re.S)
    if not m:
        raise ValueError("no LP text in test body")
    parts = re.findall(r'"((?:[^"\\]|\\.)*)"', m.group(1))
    return "".join(p.encode().decode("unicode_escape") for p in parts)


def pdhg_test_cases() -> list[dict]:
    src = open(os.path.join(REF_SRC, "tests", "test_pdhg.cpp")).read()
    cases = []
    for m in re.finditer(r"TEST\(pdhg,\s*(\w+)\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        opts = {}
        for k, v in re.findall(r"opt\.(\w+)\s*=\s*([^;]+);", body):
            opts[k] = float(v) if k.endswith("seconds") else int(float(v))
        cases.append({"name": name, "text": _c_string_literals(body), "options": opts})
    return cases


def backend_matrix() -> dict:
    src = open(os.path.join(REF_SRC, "tests", "test_l0_backend.cpp")).read()
    body = re.search(r"CsrMatrix reference_matrix\(\)\s*\{(.*?)\}\s*\n", src, re.S).group(1)
    trip = [(int(r), int(c), float(v)) for r, c, v in
            re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*,\s*([-\d.eE+]+)\s*\}", body)]
    dims = re.search(r"from_triplets\((\d+),\s*(\d+)", body)
    m, n = int(dims.group(1)), int(dims.group(2))
    rows, cols, vals = zip(*trip)
    p = pkg.Problem.from_coo(m, n, rows, cols, vals, c=np.zeros(n), col_lo=np.zeros(n),
                             col_hi=np.zeros(n), row_lo=np.zeros(m), row_hi=np.zeros(m))
    return p


def scaling_matrix() -> "pkg.Problem":
    src = open(os.path.join(REF_SRC, "tests", "test_scaling.cpp")).read()
    body = re.search(r"CsrMatrix ill_scaled\(\)\s*\{(.*?)\}\s*\n\s*\}", src, re.S).group(1)
    trip = [(int(r), int(c), float(v)) for r, c, v in
            re.findall(r"\{\s*(\d+)\s*,\s*(\d+)\s*,\s*([-\d.eE+]+)\s*\}", body)]
    dims = re.search(r"from_triplets\((\d+),\s*(\d+)", body)
    m, n = int(dims.group(1)), int(dims.group(2))
    rows, cols, vals = zip(*trip)
    return pkg.Problem.from_coo(m, n, rows, cols, vals, c=np.zeros(n), col_lo=np.zeros(n),
                                col_hi=np.zeros(n), row_lo=np.zeros(m), row_hi=np.zeros(m))


def mixed_bounds_lp(m: int, n: int, seed: int) -> "pkg.Problem":
    """Every row type (<=, >=, =, range, free) and column bound type, feasible by construction."""
    rng = np.random.default_rng(seed)
    base = pkg.lpgen.random_equality_lp(m, n, 3, seed=seed)
    x0 = rng.uniform(-2, 2, n)
    ax = pkg.lpgen.csr_matvec(base, x0)
    kind = rng.integers(0, 5, m)
    lo = np.where(kind == 0, -np.inf, ax - rng.uniform(0, 1, m))
    hi = np.where(kind == 1, np.inf, ax + rng.uniform(0, 1, m))
    lo = np.where(kind == 2, ax, lo)
    hi = np.where(kind == 2, ax, hi)
    lo = np.where(kind == 4, -np.inf, lo)
    hi = np.where(kind == 4, np.inf, hi)
    ck = rng.integers(0, 4, n)
    clo = np.where(ck == 1, -np.inf, x0 - rng.uniform(0, 3, n))
    chi = np.where(ck == 2, np.inf, x0 + rng.uniform(0, 3, n))
    clo = np.where(ck == 3, -np.inf, clo)
    chi = np.where(ck == 3, x0 + 5.0, chi)
    base.row_lo, base.row_hi, base.col_lo, base.col_hi = lo, hi, clo, chi
    base.c = rng.standard_normal(n)
    base.obj_const = 1.5
    return base


def result_arrays(r: "orc.Result", prefix: str = "ref_") -> dict:
    out = {
        prefix + "status": r.status, prefix + "objective": r.objective,
        prefix + "primal_infeasibility": r.primal_infeasibility,
        prefix + "dual_infeasibility": r.dual_infeasibility,
        prefix + "duality_gap": r.duality_gap, prefix + "iterations": r.iterations,
        prefix + "restarts": r.restarts,
        prefix + "operator_norm_estimate": r.operator_norm_estimate,
        prefix + "message": r.message, prefix + "has_point": r.primal is not None,
    }
    if r.primal is not None:
        out[prefix + "primal"] = r.primal
        out[prefix + "dual"] = r.dual
        out[prefix + "reduced_costs"] = r.reduced_costs
    return out


def save(name: str, problem, options: dict, result: "orc.Result", extra: dict | None = None):
    d = problem.to_dict() if hasattr(problem, "to_dict") else dict(problem)
    arrays = {k: np.asarray(d[k]) for k in PROBLEM_KEYS}
    arrays.update({k: np.asarray(v) for k, v in result_arrays(result).items()})
    arrays["options_json"] = np.asarray(json.dumps(options))
    if extra:
        arrays.update({k: np.asarray(v) for k, v in extra.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(f"{name:48s} {result.status:16s} it={result.iterations:8d} "
          f"restarts={result.restarts} obj={result.objective:.10g}")


def trace_digests(trace: np.ndarray) -> np.ndarray:
    """SHA-256 of each traced iterate's FP64 bytes: (iterations, 32) uint8."""
    return np.stack([np.frombuffer(hashlib.sha256(np.ascontiguousarray(row).tobytes()).digest(),
                                   dtype=np.uint8) for row in trace])


def c0_fixtures() -> None:
    """The 2,000 x 5,000 random equality LP: at tol 1e-4 (converges) and at
    the stated tol 1e-6 under the reference's default 1,000,000-iteration cap
    (ends iteration_limit: it needs about 10.6M iterations). Every one of the
    first 100 iterates is pinned by its digest; three are kept in full."""
    p0 = pkg.lpgen.random_equality_lp(2000, 5000, 5, seed=0)
    keep = [0, 9, 99]
    for name, opts in (("c0_2000x5000_tol1e-4", {"tolerance": 1e-4}),
                       ("c0_2000x5000_tol1e-6", {"tolerance": 1e-6})):
        r = orc.reference_solve(p0, trace_iters=100, **opts)
        save(name, p0, opts, r,
             {"trace_iters_kept": np.asarray(keep), "trace_x": r.trace_x[keep],
              "trace_y": r.trace_y[keep], "trace_digest_x": trace_digests(r.trace_x),
              "trace_digest_y": trace_digests(r.trace_y)})


def main() -> None:
    if not orc.ref_available():
        raise SystemExit("oracle/_ref/libsovref.so missing: run make -C oracle ref")
    if sys.argv[1:] == ["c0"]:  # only the 2,000 x 5,000 fixtures
        c0_fixtures()
        return
    # 1. the reference's PDHG unit tests (tests/test_pdhg.cpp)
    for case in pdhg_test_cases():
        d = orc.reference_read_model(case["text"])
        p = pkg.Problem.from_dict(d)
        r = orc.reference_solve(p, **case["options"])
        save("pdhg_" + case["name"], p, case["options"], r)
    # 2. the smoke models (benchmarks/smoke/*.mps), capped at 20,000 iterations
    smoke = os.path.join(REF_SRC, "benchmarks", "smoke")
    for f in sorted(os.listdir(smoke)):
        if not f.endswith(".mps"):
            continue
        d = orc.reference_read_model(open(os.path.join(smoke, f)).read(), is_mps=True)
        p = pkg.Problem.from_dict(d)
        opts = {"max_iterations": 20000}
        save("smoke_" + f[:-4], p, opts, orc.reference_solve(p, **opts))
    # 3. seeded synthetic LPs with per-iteration traces (first 100 iterations)
    synth = [
        ("rand_eq_60x150", pkg.lpgen.random_equality_lp(60, 150, 4, seed=11), {"max_iterations": 20000}),
        ("rand_eq_max_40x100", pkg.lpgen.random_equality_lp(40, 100, 3, seed=12, maximize=True),
         {"max_iterations": 20000, "tolerance": 1e-5}),
        ("mixed_bounds_50x90", mixed_bounds_lp(50, 90, 13), {"max_iterations": 6000}),
        ("mixed_bounds_period7", mixed_bounds_lp(30, 70, 14),
         {"max_iterations": 3000, "restart_check_period": 7, "tolerance": 1e-3}),
    ]
    for name, p, opts in synth:
        r = orc.reference_solve(p, trace_iters=100, **opts)
        save(name, p, opts, r, {"trace_x": r.trace_x, "trace_y": r.trace_y})
    c0_fixtures()
    # 5. backend known answers (tests/test_l0_backend.cpp) through the reference Host backend
    A = backend_matrix()
    ba = {}
    x = np.array([1.0, 2.0, 3.0])
    yv = np.array([1.0, 2.0, 3.0, 4.0])
    ba["x"], ba["y"] = x, yv
    ba["ax"] = orc.reference_spmv(A, 1.0, x, 0.0, np.zeros(4))
    ba["ax_alpha_beta"] = orc.reference_spmv(A, 2.0, x, 3.0, np.ones(4))
    ba["aty"] = orc.reference_spmv(A, 1.0, yv, 0.0, np.zeros(3), transpose=True)
    ba["ax_nan"] = orc.reference_spmv(A, 1.0, x, 0.0, np.full(4, np.nan))
    xh = np.array([0.5, -1.25, 2.75])
    ba["x_host"] = xh
    ba["ax_host"] = orc.reference_spmv(A, 1.0, xh, 0.0, np.zeros(4))
    d = A.to_dict()
    np.savez_compressed(os.path.join(HERE, "backend_known_answers.npz"),
                        **{k: np.asarray(d[k]) for k in PROBLEM_KEYS}, **ba)
    print("backend_known_answers", ba["ax"], ba["aty"])
    # 6. scaling of the reference's ill-scaled matrix (tests/test_scaling.cpp)
    S = scaling_matrix()
    rs, cs = orc.reference_scaling(S)
    rs_r, cs_r = orc.reference_scaling(S, apply_pock_chambolle=0)
    d = S.to_dict()
    np.savez_compressed(os.path.join(HERE, "scaling_ill_scaled.npz"),
                        **{k: np.asarray(d[k]) for k in PROBLEM_KEYS},
                        row_scale=rs, col_scale=cs, row_scale_ruiz=rs_r, col_scale_ruiz=cs_r)
    print("scaling_ill_scaled", rs, cs)


if __name__ == "__main__":
    main()
