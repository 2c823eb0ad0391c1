"""Long rows cut into CTA segments.

Rows longer than a work item are summed by several CTAs (or warps); the one
that finishes a row's last segment adds the segments' partials in segment
order and runs the row's update. The three long-row strategies of the
throughput kernels (CTA items above 512 entries, CTA items above 4,096, warp
items above the short rows) are pinned in turn through the tuning-cache file,
on an LP with rows of 300,000 / 100,000 / 20,000 / 4,097 entries (74, 25, 5
and 2 CTA segments; more as warp segments) beside warp-sized and short rows.
In each:

* the FP64 iterates stay within 1e-10 (relative, floor 1) of the exact
  kernels' over the first 100 iterations (no check among them, so no restart
  decision can flip);
* repeated solves, FP64 and FP32-mixed, give bit-identical results (the
  segment order fixes the sum order whatever order the CTAs finish in).
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SNIPPET = """
import importlib, json, sys
import numpy as np
sys.path.insert(0, {root!r})
pkg = importlib.import_module("sovereign-solver_b200")
lengths = [300_000, 100_000, 20_000, 4_097] + [5_000] * 10 + [3_000] * 50 + [1_000] * 400 \\
    + [600] * 200 + [8] * 3000
p = pkg.lpgen.row_lengths_lp(lengths, 400_000, seed=7)
assert p.nnz >= 1 << 20  # large enough for the tuner (and its cache) to be used

def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) if a.size else 0.0

kw = dict(max_iterations=300, tolerance=1e-12, restart_check_period=150, trace_iters=100)
with pkg.Engine(0) as e:
    e.load(p)
    ex = e.solve(pkg.PdhgOptions(**kw))
    f1 = e.solve(pkg.PdhgOptions(precision="fp64", **kw))
    f2 = e.solve(pkg.PdhgOptions(precision="fp64", **kw))
    mk = dict(precision="mixed", termination_rule="relative_kkt", restart_rule="adaptive",
              max_iterations=600, restart_check_period=40)
    m1 = e.solve(pkg.PdhgOptions(**mk))
    m2 = e.solve(pkg.PdhgOptions(**mk))
    out = dict(
        fp64=e.tuning("fp64"), mixed=e.tuning("mixed"),
        err=max(max(rel_err(f1.trace_x[k], ex.trace_x[k]), rel_err(f1.trace_y[k], ex.trace_y[k]))
                for k in range(100)),
        fp64_repeat=bool(np.array_equal(f1.primal, f2.primal) and np.array_equal(f1.dual, f2.dual)
                         and np.array_equal(f1.trace_x, f2.trace_x)),
        mixed_repeat=bool(np.array_equal(m1.primal, m2.primal) and np.array_equal(m1.dual, m2.dual)
                          and m1.objective == m2.objective),
        iterations=[ex.iterations, f1.iterations, m1.iterations])
    print(json.dumps(out))
"""


def run(cache, mode=None):
    if mode is not None:
        entries = json.loads(cache.read_text())
        cache.write_text(json.dumps({k: [v[0], mode] for k, v in entries.items()}))
    env = dict(os.environ, PDHG_B200_TUNE_CACHE=str(cache))
    r = subprocess.run([sys.executable, "-c", SNIPPET.format(root=ROOT)], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_split_rows_in_both_long_row_strategies(tmp_path):
    cache = tmp_path / "tune.json"
    runs = [(None, run(cache))]  # the tuner times the shapes and writes the file
    assert any(k.startswith("f64/dual/") for k in json.loads(cache.read_text()))
    runs += [(mode, run(cache, mode)) for mode in (0, 1, 2)]
    for mode, out in runs:
        assert out["err"] <= 1e-10, (mode, out)
        assert out["fp64_repeat"] and out["mixed_repeat"], (mode, out)
        if mode is not None:
            assert out["fp64"]["dual_long_mode"] == mode, out
            assert out["mixed"]["dual_long_mode"] == mode, out


SLICE_SNIPPET = """
import importlib, json, sys
import numpy as np
sys.path.insert(0, {root!r})
pkg = importlib.import_module("sovereign-solver_b200")
p = pkg.lpgen.transportation_lp(600, 900, seed=1000)  # 1.08M nonzeros: the tuner runs
assert p.nnz >= 1 << 20

def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) if a.size else 0.0

kw = dict(max_iterations=300, tolerance=1e-12, restart_check_period=150, trace_iters=100)
with pkg.Engine(0) as e:
    e.load(p)
    ex = e.solve(pkg.PdhgOptions(**kw))
    f1 = e.solve(pkg.PdhgOptions(precision="fp64", **kw))
    f2 = e.solve(pkg.PdhgOptions(precision="fp64", **kw))
    mk = dict(precision="mixed", termination_rule="relative_kkt", restart_rule="adaptive",
              max_iterations=200_000)
    m1 = e.solve(pkg.PdhgOptions(**mk))
    m2 = e.solve(pkg.PdhgOptions(**mk))
    f64 = e.solve(pkg.PdhgOptions(**dict(mk, precision="fp64")))
    out = dict(
        fp64=e.tuning("fp64"), mixed=e.tuning("mixed"),
        err=max(max(rel_err(f1.trace_x[k], ex.trace_x[k]), rel_err(f1.trace_y[k], ex.trace_y[k]))
                for k in range(100)),
        fp64_repeat=bool(np.array_equal(f1.primal, f2.primal) and np.array_equal(f1.dual, f2.dual)),
        mixed_repeat=bool(np.array_equal(m1.primal, m2.primal) and m1.objective == m2.objective),
        status=[m1.status, f64.status],
        obj_gap=abs(m1.objective - f64.objective) / max(1.0, abs(f64.objective)))
    print(json.dumps(out))
"""


def test_row_slices_on_a_transportation_lp(tmp_path):
    """The demand rows of a transportation LP (600 entries, consecutive rows
    gathering consecutive columns) become lane-interleaved row slices; with
    the slices pinned on (each long-row strategy for the remaining rows) and
    off, the FP64 iterates track the exact kernels, repeated solves are
    bit-identical and the mixed mode stops like the FP64 mode (at the FP64
    optimum when both converge)."""
    cache = tmp_path / "tune.json"
    env = dict(os.environ, PDHG_B200_TUNE_CACHE=str(cache))
    code = SLICE_SNIPPET.format(root=ROOT)

    def go(mode=None):
        if mode is not None:
            entries = json.loads(cache.read_text())
            cache.write_text(json.dumps(
                {k: [v[0], mode if "/dual/" in k else v[1]] for k, v in entries.items()}))
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                           text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-4000:]
        return json.loads(r.stdout.strip().splitlines()[-1])

    first = go()
    keys = json.loads(cache.read_text())
    assert any("/dual/" in k and not k.endswith("/sl0") for k in keys), keys
    for mode, out in [(None, first)] + [(m, go(m)) for m in (0, 4, 5, 6)]:
        assert out["err"] <= 1e-10, (mode, out)
        assert out["fp64_repeat"] and out["mixed_repeat"], (mode, out)
        assert out["status"][0] == out["status"][1], (mode, out)
        if out["status"][0] == "optimal":
            assert out["obj_gap"] <= 2e-3, (mode, out)
        if mode is not None:
            assert out["fp64"]["dual_long_mode"] == mode, out


def _orig_residual(p, x, y, bt):
    """The check's original-space residual of a candidate (x, y), restated in
    numpy: max over rows of the bound violation of A x and of the
    complementary-slackness term of y, and over columns of that of the
    reduced cost c - A^T y (a finite end within bt of the value is active)."""
    import numpy as np
    rows = np.repeat(np.arange(p.m), np.diff(p.row_ptr))
    act = np.zeros(p.m)
    np.add.at(act, rows, p.val * x[p.col_idx])
    aty = np.zeros(p.n)
    np.add.at(aty, p.col_idx, p.val * y[rows])
    rc = p.c - aty

    def cs(v, a, lo, hi):
        at_lo = np.isfinite(lo) & (np.abs(a - lo) < bt)
        at_hi = np.isfinite(hi) & (np.abs(a - hi) < bt)
        out = np.abs(v)
        out = np.where(at_lo & ~at_hi, np.maximum(0.0, -v), out)
        out = np.where(at_hi & ~at_lo, np.maximum(0.0, v), out)
        return np.where(at_lo & at_hi, 0.0, out)

    with np.errstate(invalid="ignore"):
        op = np.maximum(np.where(np.isfinite(p.row_lo), p.row_lo - act, 0.0),
                        np.where(np.isfinite(p.row_hi), act - p.row_hi, 0.0))
    return max(float(np.max(np.maximum(op, 0.0), initial=0.0)),
               float(np.max(cs(y, act, p.row_lo, p.row_hi), initial=0.0)),
               float(np.max(cs(rc, x, p.col_lo, p.col_hi), initial=0.0)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_check_over_row_slices_matches_the_candidates_residual(pkg, precision):
    """The check walks the demand rows of a transportation LP through their
    row slices; at every check the residual it reports for its candidate
    (the checkpoint callback's point and residual) must be the one numpy
    computes from that point."""
    import numpy as np
    p = pkg.lpgen.transportation_lp(600, 900, seed=1000)
    seen = []

    def cb(it, x, y, res):
        seen.append((it, x.copy(), y.copy(), res))

    with pkg.Engine(0) as e:
        e.load(p)
        e.solve(pkg.PdhgOptions(precision=precision, termination_rule="relative_kkt",
                                restart_rule="adaptive", max_iterations=400, tolerance=1e-4,
                                checkpoint=cb))
    assert len(seen) >= 5
    for it, x, y, res in seen:
        want = _orig_residual(p, x, y, 1e-4)
        assert res == pytest.approx(want, rel=1e-9, abs=1e-12), (it, res, want)
