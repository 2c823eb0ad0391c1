"""GPU parity: the CUDA engine, called through the C-ABI, against the
reference's outputs (golden fixtures) and the oracle on the same inputs.

* FP64-exact mode must reproduce the reference bit for bit: iterates of the
  first 100 iterations, restart counts, iteration counts, statuses, results.
* FP64 mode (warp-parallel sums): iterates within 1e-10 relative over the
  first 100 iterations, final objective within 1e-8 relative wherever both
  stop at the same iteration with the same status.
* Mixed mode (FP32 iterates, FP64 checks): same status, objective within the
  tolerance the relative-KKT rule promises.
"""
import hashlib

import numpy as np
import pytest

from conftest import PDHG_CASES, golden_problem, highs_optimum, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine(pkg):
    e = pkg.Engine(0)
    yield e
    e.close()


def solve(pkg, engine, p, **kw):
    trace = kw.pop("trace_iters", 0)
    cancel = kw.pop("cancel", None)
    x0 = kw.pop("x0", None)
    y0 = kw.pop("y0", None)
    opt = pkg.PdhgOptions(trace_iters=trace, **kw)
    engine.load(p)
    return engine.solve(opt, cancel=cancel, x0=x0, y0=y0)


def same_as_golden(r, g):
    assert r.status == g["ref_status"], (r.status, g["ref_status"], r.message)
    assert r.message == g["ref_message"]
    assert r.iterations == g["ref_iterations"]
    assert r.restarts == g["ref_restarts"]
    assert r.operator_norm_estimate == g["ref_operator_norm_estimate"]
    for f in ("objective", "primal_infeasibility", "dual_infeasibility", "duality_gap"):
        assert getattr(r, f) == g["ref_" + f], (f, getattr(r, f), g["ref_" + f])
    if g["ref_has_point"]:
        for f in ("primal", "dual", "reduced_costs"):
            assert np.array_equal(getattr(r, f), g["ref_" + f]), f


@pytest.mark.parametrize("name", PDHG_CASES)
def test_exact_mode_is_bit_identical_to_the_reference(pkg, engine, name):
    g = load_golden(name)
    p = golden_problem(pkg, g)
    tr = 100 if "trace_x" in g else 0
    r = solve(pkg, engine, p, trace_iters=tr, **g["options"])
    same_as_golden(r, g)
    if tr:
        keep = g.get("trace_iters_kept")
        tx = r.trace_x if keep is None else r.trace_x[keep]
        ty = r.trace_y if keep is None else r.trace_y[keep]
        assert np.array_equal(tx, g["trace_x"]) and np.array_equal(ty, g["trace_y"])
        if "trace_digest_x" in g:  # every one of the first 100 iterates, bit for bit
            assert np.array_equal(trace_digests(r.trace_x), g["trace_digest_x"])
            assert np.array_equal(trace_digests(r.trace_y), g["trace_digest_y"])


def trace_digests(trace):
    """SHA-256 of each traced iterate's FP64 bytes (as make_golden.py stores them)."""
    return np.stack([np.frombuffer(hashlib.sha256(np.ascontiguousarray(row).tobytes()).digest(),
                                   dtype=np.uint8) for row in trace])


def rel_err(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) if a.size else 0.0


@pytest.mark.parametrize("name", ["c0_2000x5000_tol1e-4", "c0_2000x5000_tol1e-6"])
def test_fp64_mode_tracks_all_first_100_iterates_of_the_2000x5000_lp(pkg, orc, engine, name):
    # the oracle's first 100 iterates are the reference's (their digests are
    # in the fixture); FP64 mode stays within 1e-10 of every one of them
    g = load_golden(name)
    p = golden_problem(pkg, g)
    o = orc.oracle_solve(p, trace_iters=100, max_iterations=100, **g["options"])
    assert np.array_equal(trace_digests(o.trace_x), g["trace_digest_x"])
    assert np.array_equal(trace_digests(o.trace_y), g["trace_digest_y"])
    r = solve(pkg, engine, p, precision="fp64", trace_iters=100, max_iterations=100,
              **g["options"])
    for k in range(100):
        assert rel_err(r.trace_x[k], o.trace_x[k]) <= 1e-10, k
        assert rel_err(r.trace_y[k], o.trace_y[k]) <= 1e-10, k


def test_fp64_mode_at_the_stated_tolerance_of_the_2000x5000_lp(pkg, engine):
    # tol 1e-6 under the reference's 1,000,000-iteration cap: the reference
    # ends iteration_limit there; FP64 mode must end the same way, at the same
    # iteration, with the objective within 1e-8
    g = load_golden("c0_2000x5000_tol1e-6")
    p = golden_problem(pkg, g)
    r = solve(pkg, engine, p, precision="fp64", **g["options"])
    assert r.status == g["ref_status"] == "iteration_limit"
    assert r.iterations == g["ref_iterations"] == 1_000_000
    assert abs(r.objective - g["ref_objective"]) <= 1e-8 * max(1.0, abs(g["ref_objective"]))


@pytest.mark.parametrize("name", ["rand_eq_60x150", "rand_eq_max_40x100", "mixed_bounds_50x90",
                                  "c0_2000x5000_tol1e-4"])
def test_fp64_mode_tracks_the_reference(pkg, engine, name):
    g = load_golden(name)
    p = golden_problem(pkg, g)
    r = solve(pkg, engine, p, precision="fp64", trace_iters=100, **g["options"])
    keep = g.get("trace_iters_kept")
    tx = r.trace_x if keep is None else r.trace_x[keep]
    ty = r.trace_y if keep is None else r.trace_y[keep]
    assert rel_err(tx, g["trace_x"]) <= 1e-10
    assert rel_err(ty, g["trace_y"]) <= 1e-10
    assert r.status == g["ref_status"]
    if r.iterations == g["ref_iterations"]:
        assert abs(r.objective - g["ref_objective"]) <= 1e-8 * max(1.0, abs(g["ref_objective"]))
    else:  # a decision flipped at a threshold: both must still be converged answers
        assert abs(r.iterations - g["ref_iterations"]) <= 2 * g["options"].get("restart_check_period", 40)


@pytest.mark.parametrize("name", ["rand_eq_max_40x100", "c0_2000x5000_tol1e-4",
                                  "pdhg_two_variable_optimum_matches_simplex", "smoke_tiny_lp"])
def test_mixed_mode_converges_to_the_reference_optimum(pkg, engine, name):
    g = load_golden(name)
    p = golden_problem(pkg, g)
    opts = dict(g["options"])
    r = solve(pkg, engine, p, precision="mixed", termination_rule="relative_kkt", **opts)
    assert r.status == "optimal", (r.status, r.message, r.relative_kkt)
    tol = opts.get("tolerance", 1e-4)
    assert r.relative_kkt < tol
    # |objective error| of a point with relative KKT < tol is O(tol) relative
    assert abs(r.objective - g["ref_objective"]) <= 20 * tol * (1 + abs(g["ref_objective"]))


def test_checkpoints_match_the_oracle(pkg, orc, engine):
    p = pkg.lpgen.random_equality_lp(30, 70, 3, seed=5)
    seen = []
    r = solve(pkg, engine, p, max_iterations=400, restart_check_period=50,
              checkpoint=lambda it, x, y, res: seen.append((it, x, y, res)))
    o = orc.oracle_solve(p, max_iterations=400, restart_check_period=50, checkpoints=True)
    assert [s[0] for s in seen] == [c[0] for c in o.checkpoints] == list(range(49, 400, 50))
    for a, b in zip(seen, o.checkpoints):
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[3] == b[3]
    assert r.iterations == o.iterations


def test_cancellation_and_time_limit(pkg, orc, engine):
    p = pkg.lpgen.random_equality_lp(40, 90, 4, seed=8)
    tok = pkg.CancellationToken()
    tok.cancel()
    r = solve(pkg, engine, p, cancel=tok)
    o = orc.oracle_solve(p, cancel=True)
    assert r.status == o.status == "cancelled"
    assert r.iterations == o.iterations == 0
    assert np.array_equal(r.primal, o.primal)
    r = solve(pkg, engine, p, time_limit_seconds=1e-9)
    assert r.status == "time_limit" and r.iterations == 0 and r.primal.shape == (90,)
    # a limit that fires mid-solve stops at a check-period boundary
    big = pkg.lpgen.random_equality_lp(2000, 5000, 5, seed=0)
    r = solve(pkg, engine, big, tolerance=1e-9, time_limit_seconds=0.3)
    assert r.status == "time_limit"
    assert r.iterations > 0 and r.iterations % 40 == 0
    assert r.seconds < 5.0


@pytest.mark.parametrize("mutate,msg", [
    (lambda p: p.col_lo.__setitem__(7, 11.0), "invalid problem: crossed bounds on column C7"),
    (lambda p: p.c.__setitem__(3, np.inf), "invalid problem: non-finite objective coefficient in column C3"),
    (lambda p: p.row_hi.__setitem__(2, np.nan), "invalid problem: NaN bound on row R2"),
    (lambda p: p.val.__setitem__(0, np.nan), "invalid problem: non-finite coefficient"),
    (lambda p: p.col_idx.__setitem__(1, 10_000), "invalid problem: column index out of range"),
])
def test_invalid_problems_report_like_the_reference(pkg, orc, engine, mutate, msg):
    p = pkg.lpgen.random_equality_lp(20, 50, 3, seed=6)
    mutate(p)
    r = solve(pkg, engine, p)
    o = orc.oracle_solve(p)
    assert r.status == o.status == "numerical_failure"
    assert r.message == o.message == msg
    assert r.primal.size == 0 and r.iterations == 0


def test_edge_sizes(pkg, orc, engine):
    # no iterations at all
    p = pkg.lpgen.random_equality_lp(10, 25, 2, seed=4)
    r = solve(pkg, engine, p, max_iterations=0)
    o = orc.oracle_solve(p, max_iterations=0)
    assert r.status == o.status == "iteration_limit" and r.iterations == 0
    assert np.array_equal(r.primal, o.primal) and r.objective == o.objective
    # fewer iterations than one check period (no check at all)
    r = solve(pkg, engine, p, max_iterations=17)
    o = orc.oracle_solve(p, max_iterations=17)
    assert r.iterations == o.iterations == 17 and np.array_equal(r.primal, o.primal)
    assert np.array_equal(r.dual, o.dual)
    # a problem with empty rows and columns
    q = pkg.Problem.from_coo(4, 5, [0, 0, 2], [1, 3, 3], [1.0, -2.0, 0.5], c=np.arange(5.0),
                             col_lo=np.zeros(5), col_hi=np.full(5, 3.0),
                             row_lo=np.array([-1.0, -np.inf, 0.0, 0.0]),
                             row_hi=np.array([1.0, np.inf, 1.0, 0.0]))
    r = solve(pkg, engine, q, max_iterations=500)
    o = orc.oracle_solve(q, max_iterations=500)
    assert (r.status, r.iterations, r.objective) == (o.status, o.iterations, o.objective)
    assert np.array_equal(r.primal, o.primal) and np.array_equal(r.dual, o.dual)


def test_power_iteration_early_exit_matches_the_oracle(pkg, orc, engine):
    # every row of A sums to 1 and nothing is scaled: the power iteration's
    # first w = -A u + v (u = v = 1) is zero, so the loop stops at once with
    # the estimate 0 and the step falls back (pdhg.cpp:261-265). The device
    # loop's early-exit flag must give the oracle's run bit for bit, in every
    # precision's setup.
    q = pkg.Problem.from_coo(2, 4, [0, 0, 1, 1], [0, 1, 2, 3], [0.5, 0.5, 0.25, 0.75],
                             c=np.array([1.0, 2.0, 3.0, 4.0]), col_lo=np.zeros(4),
                             col_hi=np.ones(4), row_lo=np.array([0.5, 0.5]),
                             row_hi=np.array([0.5, 0.5]))
    kw = dict(apply_ruiz=False, apply_pock_chambolle=False, max_iterations=200)
    o = orc.oracle_solve(q, **kw)
    r = solve(pkg, engine, q, **kw)
    assert r.operator_norm_estimate == o.operator_norm_estimate == 0.0
    assert (r.status, r.iterations, r.objective) == (o.status, o.iterations, o.objective)
    assert np.array_equal(r.primal, o.primal) and np.array_equal(r.dual, o.dual)
    for precision in ("mixed", "fp64"):
        assert solve(pkg, engine, q, precision=precision, **kw).operator_norm_estimate == 0.0


def test_parallel_power_iteration_is_the_estimate_up_to_rounding(pkg, orc, engine):
    # supply rows of 700 entries take the warp rows of A u; FP64-exact sums them
    # in the reference's order (bit-identical), the mixed and FP64 modes in
    # parallel partial sums, which may move the estimate by rounding only
    p = pkg.lpgen.transportation_lp(40, 700, seed=17)
    o = orc.oracle_solve(p, max_iterations=1)
    assert solve(pkg, engine, p, max_iterations=1).operator_norm_estimate == \
        o.operator_norm_estimate
    for precision in ("mixed", "fp64"):
        est = solve(pkg, engine, p, precision=precision, max_iterations=1).operator_norm_estimate
        assert abs(est - o.operator_norm_estimate) <= 1e-12 * o.operator_norm_estimate


def test_backend_known_answers(pkg):
    g = load_golden("backend_known_answers")
    A = golden_problem(pkg, g)
    assert np.array_equal(pkg.csr_spmv(A, 1.0, g["x"], 0.0, np.zeros(4)), g["ax"])
    assert np.array_equal(pkg.csr_spmv(A, 2.0, g["x"], 3.0, np.ones(4)), g["ax_alpha_beta"])
    assert np.array_equal(pkg.csr_spmv(A, 1.0, g["y"], 0.0, np.zeros(3), transpose=True), g["aty"])
    out = pkg.csr_spmv(A, 1.0, g["x"], 0.0, np.full(4, np.nan))
    assert not np.isnan(out).any() and out[1] == 18.0
    assert np.array_equal(pkg.csr_spmv(A, 1.0, g["x_host"], 0.0, np.zeros(4)), g["ax_host"])
    # project_box (tests/test_l0_backend.cpp:333-360)
    x = pkg.project_box([0.0, 0.0, -1.0, -5.0], [1.0, 10.0, 1.0, 5.0], [-3.0, 4.0, 7.0, 0.5])
    assert np.array_equal(x, [0.0, 4.0, 1.0, 0.5])
    x = pkg.project_box([0.0, 0.0], None, [-3.0, 1e9])
    assert np.array_equal(x, [0.0, 1e9])


def test_spmv_matches_the_oracle_on_a_large_badly_scaled_matrix(pkg, orc):
    p = pkg.lpgen.badly_scaled_lp(3000, 8000, 6, seed=21)
    x = np.random.default_rng(0).standard_normal(p.n)
    y = np.random.default_rng(1).standard_normal(p.m)
    assert np.array_equal(pkg.csr_spmv(p, -1.0, x, 0.0, np.zeros(p.m)),
                          orc.oracle_spmv(p, -1.0, x, 0.0, np.zeros(p.m)))
    assert np.array_equal(pkg.csr_spmv(p, 0.5, y, 2.0, np.ones(p.n), transpose=True),
                          orc.oracle_spmv(p, 0.5, y, 2.0, np.ones(p.n), transpose=True))


def test_exact_mode_on_a_power_law_lp_matches_the_oracle(pkg, orc, engine):
    # long rows (> 512 nonzeros) exercise the one-CTA-per-row paths
    p = pkg.lpgen.badly_scaled_lp(1500, 4000, 6, seed=22)
    r = solve(pkg, engine, p, max_iterations=400, tolerance=1e-6)
    o = orc.oracle_solve(p, max_iterations=400, tolerance=1e-6)
    assert (r.status, r.iterations, r.restarts) == (o.status, o.iterations, o.restarts)
    assert np.array_equal(r.primal, o.primal) and np.array_equal(r.dual, o.dual)
    assert r.objective == o.objective


def test_fp64_mode_on_a_power_law_lp_tracks_exact_mode(pkg, engine):
    # long rows (> 512 nonzeros) through the warp-parallel FP64 kernels: the
    # first 100 iterates stay within FP64 rounding of the exact ones
    p = pkg.lpgen.badly_scaled_lp(1500, 4000, 6, seed=22)
    ex = solve(pkg, engine, p, max_iterations=400, tolerance=1e-6, trace_iters=100)
    r2 = solve(pkg, engine, p, precision="fp64", max_iterations=400, tolerance=1e-6,
               trace_iters=100)
    errs_x = [rel_err(r2.trace_x[k], ex.trace_x[k]) for k in range(100)]
    errs_y = [rel_err(r2.trace_y[k], ex.trace_y[k]) for k in range(100)]
    first_bad = next((k for k in range(100) if max(errs_x[k], errs_y[k]) > 1e-10), None)
    assert first_bad is None, (first_bad, errs_x[first_bad], errs_y[first_bad], ex.restarts,
                               r2.restarts)
    assert r2.iterations == ex.iterations


def test_fp64_mode_tracks_exact_mode_across_row_tiers(pkg, engine):
    # rows of 8 (lane groups), 600 and 3,000 (one warp) and 20,000 nonzeros
    # (one CTA): the FP64 iterates stay within 1e-10 of the exact ones over
    # the first 100 iterations (no check among them, so no restart decision
    # can flip), and mixed mode converges to the same optimum
    p = pkg.lpgen.row_lengths_lp([20_000] + [3_000] * 4 + [600] * 20 + [8] * 200, 25_000, seed=5)
    kw = dict(max_iterations=300, tolerance=1e-12, restart_check_period=150)
    ex = solve(pkg, engine, p, trace_iters=100, **kw)
    r2 = solve(pkg, engine, p, precision="fp64", trace_iters=100, **kw)
    for k in range(100):
        assert rel_err(r2.trace_x[k], ex.trace_x[k]) <= 1e-10, k
        assert rel_err(r2.trace_y[k], ex.trace_y[k]) <= 1e-10, k
    full = dict(termination_rule="relative_kkt", restart_rule="adaptive", max_iterations=200_000)
    r64 = solve(pkg, engine, p, precision="fp64", **full)
    r32 = solve(pkg, engine, p, precision="mixed", **full)
    assert r64.status == r32.status == "optimal"
    assert abs(r32.objective - r64.objective) <= 2e-3 * max(1.0, abs(r64.objective))


def test_device_scaling_is_the_reference_scaling(pkg, orc, engine):
    for p in (pkg.lpgen.badly_scaled_lp(1500, 4000, 6, seed=22),
              pkg.lpgen.random_equality_lp(300, 700, 5, seed=2),
              golden_problem(pkg, load_golden("scaling_ill_scaled"))):
        engine.load(p)
        rs, cs = engine.scaling()
        ors, ocs = orc.oracle_scaling(p)
        assert np.array_equal(rs, ors) and np.array_equal(cs, ocs)
    # non-default scaling options rescale on the device at solve time
    p = pkg.lpgen.badly_scaled_lp(800, 2000, 5, seed=23)
    engine.load(p)
    for kw in ({"apply_pock_chambolle": False}, {"apply_ruiz": False}, {"ruiz_iterations": 2}):
        engine.solve(pkg.PdhgOptions(max_iterations=0, **kw))
        rs, cs = engine.scaling()
        ors, ocs = orc.oracle_scaling(p, **{k: int(v) for k, v in kw.items()})
        assert np.array_equal(rs, ors) and np.array_equal(cs, ocs), kw


def test_entries_dropped_by_scaling_match_the_reference(pkg, orc, engine):
    # a coefficient that scaling drives to |v| <= 1e-14 leaves the scaled matrix
    # (the reference's from_triplets rebuild drops it, src/l0/sparse.cpp:55)
    p = pkg.Problem.from_coo(3, 3, [0, 0, 1, 1, 2, 2], [0, 1, 1, 2, 0, 2],
                             [1e6, 1e-14, 2.0, 1.0, 3.0, 1e-9], c=np.array([1.0, -1.0, 0.5]),
                             col_lo=np.zeros(3), col_hi=np.full(3, 5.0),
                             row_lo=np.array([-1.0, 0.0, 1.0]), row_hi=np.array([2.0, 3.0, 4.0]))
    r = solve(pkg, engine, p, max_iterations=2000)
    o = orc.oracle_solve(p, max_iterations=2000)
    assert (r.status, r.iterations, r.restarts) == (o.status, o.iterations, o.restarts)
    assert np.array_equal(r.primal, o.primal) and np.array_equal(r.dual, o.dual)
    assert r.objective == o.objective


def test_transportation_lp_adaptive_restarts(pkg, orc, engine):
    # the reference rule never restarts here (its oracle run stalls); the
    # adaptive rule solves it, and FP64 mode follows the oracle's restatement
    p = pkg.lpgen.transportation_lp(40, 100, seed=1000)
    kw = dict(termination_rule="relative_kkt", restart_rule="adaptive", max_iterations=200_000)
    o = orc.oracle_solve(p, termination_rule=1, restart_rule=1, max_iterations=200_000)
    assert o.status == "optimal"
    r64 = solve(pkg, engine, p, precision="fp64", **kw)
    assert r64.status == "optimal"
    assert abs(r64.iterations - o.iterations) <= 200 and abs(r64.restarts - o.restarts) <= 2
    assert abs(r64.objective - o.objective) <= 1e-4 * abs(o.objective)
    r = solve(pkg, engine, p, precision="mixed", **kw)
    assert r.status == "optimal", (r.status, r.relative_kkt, r.iterations)
    assert r.relative_kkt < 1e-4
    assert abs(r.objective - o.objective) <= 2e-3 * abs(o.objective)


@pytest.mark.parametrize("seed", [3, 4])
def test_fp64_adaptive_and_primal_weight_follow_the_oracle(pkg, orc, engine, seed):
    p = pkg.lpgen.random_equality_lp(200, 500, 5, seed=seed)
    for pw in (0, 1):
        o = orc.oracle_solve(p, termination_rule=1, restart_rule=1, primal_weight_update=pw,
                             max_iterations=100_000)
        r = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt",
                  restart_rule="adaptive", primal_weight_update=bool(pw), max_iterations=100_000)
        assert r.status == o.status == "optimal"
        assert r.restarts == o.restarts and r.iterations == o.iterations, (r.iterations, o.iterations)
        assert abs(r.objective - o.objective) <= 1e-8 * abs(o.objective)


RULE2_CASES = {"equality_200x500": ("random_equality_lp", (200, 500, 5), dict(seed=3)),
               "badly_scaled_300x800": ("badly_scaled_lp", (300, 800, 5), dict(seed=2001)),
               "transportation_40x100": ("transportation_lp", (40, 100), dict(seed=1000)),
               "maximize_80x200": ("random_equality_lp", (80, 200, 4), dict(seed=8, maximize=True))}


@pytest.mark.parametrize("name", sorted(RULE2_CASES))
def test_fp64_rule2_follows_the_oracle(pkg, orc, engine, name):
    # termination rule 2 (PDLP's relative KKT) with restart rule 2 on its
    # measure: FP64 mode takes the oracle's restarts and stops where it stops
    fn, args, kw = RULE2_CASES[name]
    p = getattr(pkg.lpgen, fn)(*args, **kw)
    for pw in (0, 1):
        o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=pw,
                             max_iterations=200_000)
        r = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt_l2",
                  restart_rule="adaptive_l2", primal_weight_update=bool(pw),
                  max_iterations=200_000)
        assert r.status == o.status == "optimal", (pw, r.status, o.status)
        assert abs(r.iterations - o.iterations) <= 40 and abs(r.restarts - o.restarts) <= 1, \
            (pw, r.iterations, o.iterations, r.restarts, o.restarts)
        if r.iterations == o.iterations:
            assert abs(r.objective - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
            assert r.relative_kkt == pytest.approx(o.relative_kkt, rel=1e-8, abs=1e-14)
        assert r.relative_kkt < 1e-4


@pytest.mark.parametrize("name", sorted(RULE2_CASES))
def test_mixed_rule2_reaches_the_fp64_optimum(pkg, orc, engine, name):
    fn, args, kw = RULE2_CASES[name]
    p = getattr(pkg.lpgen, fn)(*args, **kw)
    o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=1,
                         max_iterations=200_000)
    r = solve(pkg, engine, p, precision="mixed", termination_rule="relative_kkt_l2",
              restart_rule="adaptive_l2", primal_weight_update=True, max_iterations=200_000)
    assert r.status == "optimal", (r.status, r.relative_kkt, r.iterations)
    assert r.relative_kkt < 1e-4
    # a point at 1e-4 relative KKT has its objective within about 1e-3 of the
    # optimum (HiGHS); the oracle's own FP64 point meets the same bound
    opt = highs_optimum(p)
    assert abs(r.objective - opt) <= 2e-3 * (1 + abs(opt)), (r.objective, opt)
    assert abs(o.objective - opt) <= 2e-3 * (1 + abs(opt)), (o.objective, opt)


@pytest.mark.parametrize("name", sorted(RULE2_CASES))
def test_fp64_halpern_follows_the_oracle(pkg, orc, engine, name):
    # the reflected restarted Halpern iteration: FP64 mode takes the oracle's
    # restarts and stops where it stops, reporting T(z)
    fn, args, kw = RULE2_CASES[name]
    p = getattr(pkg.lpgen, fn)(*args, **kw)
    for pw in (0, 1):
        o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=pw,
                             halpern=1, max_iterations=200_000)
        r = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt_l2",
                  restart_rule="adaptive_l2", primal_weight_update=bool(pw), halpern=True,
                  max_iterations=200_000)
        assert r.status == o.status == "optimal", (pw, r.status, o.status)
        assert abs(r.iterations - o.iterations) <= 40 and abs(r.restarts - o.restarts) <= 1, \
            (pw, r.iterations, o.iterations, r.restarts, o.restarts)
        if r.iterations == o.iterations:
            assert abs(r.objective - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
        assert r.relative_kkt < 1e-4
        assert np.all(r.primal >= p.col_lo - 1e-9) and np.all(r.primal <= p.col_hi + 1e-9)


@pytest.mark.parametrize("name", sorted(RULE2_CASES))
def test_mixed_halpern_reaches_the_fp64_optimum(pkg, orc, engine, name):
    fn, args, kw = RULE2_CASES[name]
    p = getattr(pkg.lpgen, fn)(*args, **kw)
    o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=1,
                         max_iterations=200_000)
    r = solve(pkg, engine, p, precision="mixed", termination_rule="relative_kkt_l2",
              restart_rule="adaptive_l2", primal_weight_update=True, halpern=True,
              max_iterations=200_000)
    assert r.status == "optimal", (r.status, r.relative_kkt, r.iterations)
    assert r.relative_kkt < 1e-4
    opt = highs_optimum(p)
    assert abs(r.objective - opt) <= 2e-3 * (1 + abs(opt)), (r.objective, opt)
    assert abs(o.objective - opt) <= 2e-3 * (1 + abs(opt)), (o.objective, opt)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("max_it", [200_000, 97, 23])
@pytest.mark.parametrize("name", ["transportation_40x100", "badly_scaled_300x800"])
def test_lean_halpern_is_the_stored_form(pkg, engine, precision, max_it, name):
    # Without a trace the Halpern iteration stores no z: the primal pass
    # rebuilds x from x_bar and the anchor, and T(z) is stored only where a
    # check or the result reads it (97: a tail after two checks; 23: no check
    # at all). A trace switches to the stored form. Same kernels' arithmetic,
    # so the same point bit for bit.
    fn, args, kw = RULE2_CASES[name]
    p = getattr(pkg.lpgen, fn)(*args, **kw)
    o = dict(precision=precision, termination_rule="relative_kkt_l2", restart_rule="adaptive_l2",
             primal_weight_update=True, halpern=True, max_iterations=max_it)
    lean = solve(pkg, engine, p, **o)
    full = solve(pkg, engine, p, trace_iters=1, **o)
    assert (lean.status, lean.iterations, lean.restarts) == \
        (full.status, full.iterations, full.restarts)
    assert lean.fp64_iterations == full.fp64_iterations
    np.testing.assert_array_equal(lean.primal, full.primal)
    np.testing.assert_array_equal(lean.dual, full.dual)
    assert lean.objective == full.objective


@pytest.mark.parametrize("lp", [("random_equality_lp", (200, 500, 4), dict(seed=31)),
                                ("badly_scaled_lp", (300, 800, 8), dict(seed=2002)),
                                ("random_equality_lp", (150, 400, 2), dict(seed=32))])
def test_uniform_rows_follow_the_oracle(pkg, orc, engine, lp):
    # every column with 2, 4 or 8 entries: the primal pass runs the persistent
    # uniform-row kernel (one vector load of indices and of values per lane,
    # the next row's loads in flight during the current row's gathers)
    fn, args, kw = lp
    p = getattr(pkg.lpgen, fn)(*args, **kw)
    per_col = np.bincount(p.col_idx, minlength=p.n)
    assert np.all(per_col == args[2])
    o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=1,
                         halpern=1, max_iterations=200_000)
    r = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt_l2",
              restart_rule="adaptive_l2", primal_weight_update=True, halpern=True,
              max_iterations=200_000)
    assert r.status == o.status == "optimal", (r.status, o.status)
    assert abs(r.iterations - o.iterations) <= 40, (r.iterations, o.iterations)
    if r.iterations == o.iterations:
        assert abs(r.objective - o.objective) <= 1e-8 * max(1.0, abs(o.objective))
    m = solve(pkg, engine, p, precision="mixed", termination_rule="relative_kkt_l2",
              restart_rule="adaptive_l2", primal_weight_update=True, halpern=True,
              max_iterations=200_000)
    assert m.status == "optimal" and m.relative_kkt < 1e-4
    opt = highs_optimum(p)
    assert abs(m.objective - opt) <= 2e-3 * (1 + abs(opt)), (m.objective, opt)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("demands", [400, 2000])
def test_dense_rows_match_loaded_columns(pkg, engine, monkeypatch, precision, demands):
    # The supply rows of a transportation LP sit in consecutive columns: the
    # long-row paths compute those columns instead of loading them (400
    # entries: one warp per row; 2,000: CTA items). The sum order is the
    # same, so the solve matches the one that loads every index bit for bit.
    p = pkg.lpgen.transportation_lp(40, demands, seed=1000)
    o = dict(precision=precision, termination_rule="relative_kkt_l2", restart_rule="adaptive_l2",
             primal_weight_update=True, halpern=True, max_iterations=3000)
    dense = solve(pkg, engine, p, **o)
    monkeypatch.setenv("PDHG_B200_DENSE_ROWS", "0")
    loaded = solve(pkg, engine, p, **o)
    assert (dense.status, dense.iterations, dense.restarts) == \
        (loaded.status, loaded.iterations, loaded.restarts)
    np.testing.assert_array_equal(dense.primal, loaded.primal)
    np.testing.assert_array_equal(dense.dual, loaded.dual)


@pytest.mark.parametrize("halpern", [False, True])
def test_fp64_warm_start_follows_the_oracle(pkg, orc, engine, halpern):
    # x0 / y0 (original units): x = proj(x0 / col_scale), y = y0 sign / row_scale,
    # s = proj(A x); the oracle restates the same start
    p = pkg.lpgen.random_equality_lp(200, 500, 5, seed=21)
    kw = dict(termination_rule=2, restart_rule=2, primal_weight_update=1, halpern=int(halpern),
              max_iterations=200_000)
    base = orc.oracle_solve(p, **kw)
    rng = np.random.default_rng(5)
    x0 = base.primal * (1 + 0.05 * rng.standard_normal(p.n))
    y0 = base.dual * (1 + 0.05 * rng.standard_normal(p.m))
    o = orc.oracle_solve(p, x0=x0, y0=y0, **kw)
    r = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt_l2",
              restart_rule="adaptive_l2", primal_weight_update=True, halpern=halpern,
              max_iterations=200_000, x0=x0, y0=y0)
    assert r.status == o.status == "optimal"
    assert abs(r.iterations - o.iterations) <= 40, (r.iterations, o.iterations)
    if r.iterations == o.iterations:
        assert abs(r.objective - o.objective) <= 1e-8 * max(1.0, abs(o.objective))


def test_halpern_option_combinations_are_checked(pkg, engine):
    p = pkg.lpgen.random_equality_lp(20, 50, 3, seed=1)
    with pytest.raises(pkg.PdhgError):  # needs rule 2 and restart rule 2
        solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt",
              restart_rule="adaptive", halpern=True)
    with pytest.raises(pkg.PdhgError):  # not in the reference's exact mode
        solve(pkg, engine, p, termination_rule="relative_kkt_l2", restart_rule="adaptive_l2",
              halpern=True)


def test_rule2_option_combinations_are_checked(pkg, engine):
    p = pkg.lpgen.random_equality_lp(20, 50, 3, seed=1)
    with pytest.raises(pkg.PdhgError):  # rule 2 needs mixed or fp64
        solve(pkg, engine, p, termination_rule="relative_kkt_l2")
    with pytest.raises(pkg.PdhgError):  # restart rule 2 restarts on rule 2's measure
        solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt",
              restart_rule="adaptive_l2")


def test_exact_mode_rejects_the_extensions(pkg, engine):
    p = pkg.lpgen.random_equality_lp(20, 50, 3, seed=1)
    with pytest.raises(pkg.PdhgError):
        solve(pkg, engine, p, restart_rule="adaptive")


def test_warm_start_from_the_solution_converges_immediately(pkg, engine):
    p = pkg.lpgen.random_equality_lp(60, 150, 4, seed=30)
    cold = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt",
                 max_iterations=200_000)
    assert cold.status == "optimal"
    warm = solve(pkg, engine, p, precision="fp64", termination_rule="relative_kkt",
                 max_iterations=200_000, x0=cold.primal, y0=cold.dual)
    assert warm.status == "optimal"
    assert warm.iterations < cold.iterations


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_feed_matches_the_synchronous_copies(pkg, engine, precision):
    # with a callback the engine keeps two periods in flight and hands each
    # candidate over through a pinned slot; verbose output keeps one period in
    # flight and copies synchronously: both must deliver the same calls
    p = pkg.lpgen.random_equality_lp(300, 800, 5, seed=31)
    runs = []
    for verbose in (False, True):
        seen = []
        r = solve(pkg, engine, p, precision=precision, max_iterations=2000, tolerance=1e-7,
                  termination_rule="relative_kkt", restart_rule="adaptive", verbose=verbose,
                  checkpoint=lambda it, x, y, res: seen.append((it, x, y, res)))
        runs.append((r, seen))
    (r1, s1), (r2, s2) = runs
    assert [s[0] for s in s1] == [s[0] for s in s2] and len(s1) > 5
    assert [s[0] for s in s1] == list(range(39, 40 * len(s1), 40))
    for a, b in zip(s1, s2):
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[3] == b[3]
    assert (r1.status, r1.iterations, r1.objective) == (r2.status, r2.iterations, r2.objective)
