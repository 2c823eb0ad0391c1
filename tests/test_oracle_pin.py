"""Pins the oracle (plain-C restatement) to the reference itself.

oracle/_ref/libsovref.so is the reference's own PDHG path compiled from its
sources (oracle/Makefile). On identical inputs the restatement must reproduce
it bit for bit: iterates, restarts, statuses, every result field.
"""
import numpy as np
import pytest

from conftest import golden_problem, load_golden

pytestmark = pytest.mark.filterwarnings("ignore")


def _ref_or_skip(orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")


def _same(a, b):
    assert a.status == b.status, (a.status, b.status, a.message, b.message)
    assert a.message == b.message
    assert a.iterations == b.iterations
    assert a.restarts == b.restarts
    for f in ("objective", "primal_infeasibility", "dual_infeasibility", "duality_gap",
              "operator_norm_estimate"):
        va, vb = getattr(a, f), getattr(b, f)
        assert va == vb or (np.isnan(va) and np.isnan(vb)), (f, va, vb)
    for f in ("primal", "dual", "reduced_costs"):
        va, vb = getattr(a, f), getattr(b, f)
        assert (va is None) == (vb is None)
        if va is not None:
            assert np.array_equal(va, vb), f


@pytest.mark.parametrize("seed,maximize", [(1, False), (2, True), (3, False)])
def test_oracle_is_the_reference_on_random_lps(pkg, orc, seed, maximize):
    _ref_or_skip(orc)
    p = pkg.lpgen.random_equality_lp(40, 90, 4, seed=seed, maximize=maximize)
    kw = dict(max_iterations=4000, trace_iters=30)
    a, b = orc.oracle_solve(p, **kw), orc.reference_solve(p, **kw)
    _same(a, b)
    assert np.array_equal(a.trace_x, b.trace_x) and np.array_equal(a.trace_y, b.trace_y)


def test_oracle_is_the_reference_with_restarts_and_every_bound_type(pkg, orc):
    _ref_or_skip(orc)
    g = load_golden("mixed_bounds_50x90")
    p = golden_problem(pkg, g)
    for kw in (dict(max_iterations=3000), dict(max_iterations=2000, restart_check_period=3,
                                                restart_sufficient_decrease=0.9)):
        _same(orc.oracle_solve(p, **kw), orc.reference_solve(p, **kw))


def test_checkpoints_match(pkg, orc):
    _ref_or_skip(orc)
    p = pkg.lpgen.random_equality_lp(30, 70, 3, seed=5)
    a = orc.oracle_solve(p, max_iterations=400, restart_check_period=50, checkpoints=True)
    b = orc.reference_solve(p, max_iterations=400, restart_check_period=50, checkpoints=True)
    assert [c[0] for c in a.checkpoints] == [c[0] for c in b.checkpoints] == list(range(49, 400, 50))
    for ca, cb in zip(a.checkpoints, b.checkpoints):
        assert np.array_equal(ca[1], cb[1]) and np.array_equal(ca[2], cb[2]) and ca[3] == cb[3]


def test_time_limit_and_invalid_input_match(pkg, orc):
    _ref_or_skip(orc)
    p = pkg.lpgen.random_equality_lp(20, 50, 3, seed=6)
    _same(orc.oracle_solve(p, time_limit_seconds=1e-9), orc.reference_solve(p, time_limit_seconds=1e-9))
    bad = pkg.lpgen.random_equality_lp(20, 50, 3, seed=6)
    bad.col_lo[7] = 11.0  # crossed: lo > hi = 10
    _same(orc.oracle_solve(bad), orc.reference_solve(bad))
    bad2 = pkg.lpgen.random_equality_lp(20, 50, 3, seed=6)
    bad2.c[3] = np.inf
    _same(orc.oracle_solve(bad2), orc.reference_solve(bad2))
    bad3 = pkg.lpgen.random_equality_lp(20, 50, 3, seed=6)
    bad3.row_hi[2] = np.nan
    _same(orc.oracle_solve(bad3), orc.reference_solve(bad3))


def test_scaling_and_spmv_match(pkg, orc):
    _ref_or_skip(orc)
    p = pkg.lpgen.badly_scaled_lp(300, 700, 5, seed=9)
    for kw in ({}, {"apply_ruiz": 0}, {"apply_pock_chambolle": 0}, {"ruiz_iterations": 3}):
        ra, ca = orc.oracle_scaling(p, **kw)
        rb, cb = orc.reference_scaling(p, **kw)
        assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
    x = np.random.default_rng(0).standard_normal(p.n)
    y = np.random.default_rng(1).standard_normal(p.m)
    assert np.array_equal(orc.oracle_spmv(p, -1.0, x, 0.0, np.zeros(p.m)),
                          orc.reference_spmv(p, -1.0, x, 0.0, np.zeros(p.m)))
    assert np.array_equal(orc.oracle_spmv(p, 0.5, y, 2.0, np.ones(p.n), transpose=True),
                          orc.reference_spmv(p, 0.5, y, 2.0, np.ones(p.n), transpose=True))


def _same_ranges(a, b):
    for u, v in zip(a, b):
        assert u == v or (np.isnan(u) and np.isnan(v)), (a, b)


def test_certificate_checker_is_the_reference(pkg, orc):
    # FarkasCertificate{y}.certifies_infeasibility (src/l1/duals.cpp:16-79):
    # verdict and both ranges, bit for bit, on the reference's infeasible
    # smoke model (x >= 0, x >= 2, x <= 1: y = (1, -1) certifies it) and on
    # random multipliers over random LPs (zero multipliers included)
    _ref_or_skip(orc)
    p = golden_problem(pkg, load_golden("smoke_tiny_infeasible"))
    for y, expect in (([1.0, -1.0], True), ([1.0, 1.0], False), ([0.0, 0.0], False)):
        a, ra = orc.oracle_certifies(p, y)
        b, rb = orc.reference_certifies(p, y)
        assert a == b == expect
        _same_ranges(ra, rb)
    rng = np.random.default_rng(5)
    for seed in range(4):
        q = pkg.lpgen.badly_scaled_lp(40, 90, 4, seed=seed)
        for _ in range(5):
            y = rng.standard_normal(q.m) * (rng.random(q.m) < 0.7)
            a, ra = orc.oracle_certifies(q, y)
            b, rb = orc.reference_certifies(q, y)
            assert a == b
            _same_ranges(ra, rb)
    # with the lower bound of the first row dropped the row side becomes
    # (-inf, inf): nothing is certified
    q = golden_problem(pkg, load_golden("smoke_tiny_infeasible"))
    q.row_lo = np.array([-np.inf, -np.inf])
    a, ra = orc.oracle_certifies(q, [1.0, -1.0])
    b, rb = orc.reference_certifies(q, [1.0, -1.0])
    assert a == b is False
    _same_ranges(ra, rb)


def test_ray_checker_on_known_rays(pkg, orc):
    # the engine's dual-infeasibility ray test (no reference counterpart),
    # restated in numpy, on the reference's unbounded smoke model
    # (min -x1, x1 - x2 <= 5, x >= 0: d = (1, 1) keeps every bound and the
    # objective falls by 1 along it)
    p = golden_problem(pkg, load_golden("smoke_tiny_unbounded"))
    ok, obj, viol = orc.ray_certifies(p, [2.0, 2.0])  # scaled to max |d| = 1
    assert ok and obj == -1.0 and viol == 0.0
    ok, obj, viol = orc.ray_certifies(p, [1.0, 0.0])  # x1 - x2 grows past its upper end
    assert not ok and viol == 1.0
    ok, obj, viol = orc.ray_certifies(p, [-1.0, -1.0])  # leaves x >= 0, objective rises
    assert not ok and obj == 1.0
    assert not orc.ray_certifies(p, [0.0, 0.0])[0]
    assert not orc.ray_certifies(p, [np.nan, 1.0])[0]
    # within eps of the cone (1e-7 above the row's end, objective -1): certified
    assert orc.ray_certifies(p, [1.0, 1.0 - 1e-7])[0]
    assert not orc.ray_certifies(p, [1.0, 1.0 - 1e-5])[0]
    # maximize: max x1 is the same ray
    q = golden_problem(pkg, load_golden("smoke_tiny_unbounded"))
    q.c, q.maximize = np.array([1.0, 0.0]), True
    ok, obj, _ = orc.ray_certifies(q, [1.0, 1.0])
    assert ok and obj == -1.0
    # a bounded LP (columns boxed) has no ray
    b = pkg.lpgen.random_equality_lp(30, 70, 3, seed=5)
    rng = np.random.default_rng(3)
    assert not any(orc.ray_certifies(b, rng.standard_normal(b.n))[0] for _ in range(20))
