"""The batched engine (pdhg_load_batch / pdhg_solve_batch) through the C-ABI.

Every instance of a batch must come out as its own solve would: the oracle's
restatement of Pdhg::solve run on that instance alone is the reference. FP64
mode follows the oracle's iteration and restart counts; mixed mode reaches the
oracle's optimum within the relative-KKT tolerance. Invalid instances, limits,
cancellation and warm starts behave per instance like the single engine.
"""
import dataclasses

import numpy as np
import pytest

from conftest import golden_problem, load_golden

pytestmark = pytest.mark.gpu

ADAPTIVE = dict(termination_rule="relative_kkt", restart_rule="adaptive")


@pytest.fixture(scope="module")
def engine(pkg):
    e = pkg.Engine(0)
    yield e
    e.close()


def family(pkg):
    """Instances of uneven size and kind, each solved by the oracle under the
    adaptive rule: equality rows, badly scaled inequality rows with box
    bounds, a transportation LP, a maximize instance with an objective
    constant."""
    q = golden_problem(pkg, load_golden("rand_eq_max_40x100"))
    return [pkg.lpgen.random_equality_lp(40, 100, 4, seed=11),
            pkg.lpgen.random_equality_lp(120, 300, 6, seed=12),
            pkg.lpgen.badly_scaled_lp(60, 150, 4, seed=7),
            pkg.lpgen.random_equality_lp(15, 45, 3, seed=13),
            pkg.lpgen.transportation_lp(10, 20, seed=5),
            dataclasses.replace(q, obj_const=3.25)]


def test_batch_fp64_follows_the_oracle_per_instance(pkg, orc, engine):
    ps = family(pkg)
    engine.load_batch(ps)
    rs = engine.solve_batch(pkg.PdhgOptions(precision="fp64", max_iterations=100_000, **ADAPTIVE))
    for k, (p, r) in enumerate(zip(ps, rs)):
        o = orc.oracle_solve(p, termination_rule=1, restart_rule=1, max_iterations=100_000)
        assert r.status == o.status == "optimal", (k, r.status, o.status, r.message)
        assert abs(r.iterations - o.iterations) <= 80 and abs(r.restarts - o.restarts) <= 1, \
            (k, r.iterations, o.iterations, r.restarts, o.restarts)
        assert abs(r.objective - o.objective) <= 1e-6 * max(1.0, abs(o.objective)), \
            (k, r.objective, o.objective)
        assert r.primal.shape == (p.n,) and r.dual.shape == (p.m,)
        assert abs(r.operator_norm_estimate - o.operator_norm_estimate) <= \
            1e-12 * o.operator_norm_estimate


def test_batch_rule2_follows_the_oracle_per_instance(pkg, orc, engine):
    ps = family(pkg)
    engine.load_batch(ps)
    for prec in ("fp64", "mixed"):
        rs = engine.solve_batch(pkg.PdhgOptions(
            precision=prec, max_iterations=200_000, termination_rule="relative_kkt_l2",
            restart_rule="adaptive_l2", primal_weight_update=True))
        for k, (p, r) in enumerate(zip(ps, rs)):
            o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=1,
                                 max_iterations=200_000)
            assert r.status == o.status == "optimal", (prec, k, r.status, o.status, r.message)
            assert r.relative_kkt < 1e-4
            if prec == "fp64":
                assert abs(r.iterations - o.iterations) <= 80, (k, r.iterations, o.iterations)
            assert abs(r.objective - o.objective) <= 1e-3 * (1 + abs(o.objective)), \
                (prec, k, r.objective, o.objective)


def test_batch_halpern_follows_the_oracle_per_instance(pkg, orc, engine):
    ps = family(pkg)
    engine.load_batch(ps)
    for prec in ("fp64", "mixed"):
        rs = engine.solve_batch(pkg.PdhgOptions(
            precision=prec, max_iterations=200_000, termination_rule="relative_kkt_l2",
            restart_rule="adaptive_l2", primal_weight_update=True, halpern=True))
        for k, (p, r) in enumerate(zip(ps, rs)):
            o = orc.oracle_solve(p, termination_rule=2, restart_rule=2, primal_weight_update=1,
                                 halpern=1, max_iterations=200_000)
            assert r.status == o.status == "optimal", (prec, k, r.status, o.status, r.message)
            assert r.relative_kkt < 1e-4
            if prec == "fp64":
                assert abs(r.iterations - o.iterations) <= 80, (k, r.iterations, o.iterations)
            assert abs(r.objective - o.objective) <= 1e-3 * (1 + abs(o.objective)), \
                (prec, k, r.objective, o.objective)


def test_batch_autotuner_keeps_the_answers(pkg, engine):
    # a batch above the tuner's 2^20-nonzero threshold: the tuned lane widths
    # must give the untuned solve's answers (mixed precision, to the rule's
    # tolerance; the width changes only the order of FP32 sums)
    ps = pkg.lpgen.batch_family(96, seed_base=3000, m_lo=2000, m_hi=5000)
    assert sum(p.nnz for p in ps) >= 1 << 20
    opt = dict(precision="mixed", max_iterations=200_000, termination_rule="relative_kkt_l2",
               restart_rule="adaptive_l2", primal_weight_update=True)
    engine.load_batch(ps)
    fixed = engine.solve_batch(pkg.PdhgOptions(autotune=False, **opt), want_point=False)
    t0 = engine.batch_tuning("mixed")
    assert not t0["timed"]
    tuned = engine.solve_batch(pkg.PdhgOptions(**opt), want_point=False)
    t1 = engine.batch_tuning("mixed")
    assert t1["timed"]
    for lanes in (t1["primal_lanes"], t1["dual_lanes"]):
        assert lanes in (1, 2, 4, 8, 16, 32)
    for k, (a, b) in enumerate(zip(fixed, tuned)):
        assert a.status == b.status == "optimal", (k, a.status, b.status)
        assert b.relative_kkt < 1e-4
        assert abs(a.objective - b.objective) <= 1e-3 * (1 + abs(a.objective)), k
    again = engine.solve_batch(pkg.PdhgOptions(**opt), want_point=False)
    assert engine.batch_tuning("mixed") == t1  # kept until the next load
    assert [r.iterations for r in again] == [r.iterations for r in tuned]


def test_batch_mixed_solves_every_instance(pkg, orc, engine):
    ps = family(pkg)
    engine.load_batch(ps)
    rs = engine.solve_batch(pkg.PdhgOptions(precision="mixed", max_iterations=200_000,
                                            **ADAPTIVE))
    for k, (p, r) in enumerate(zip(ps, rs)):
        o = orc.oracle_solve(p, termination_rule=1, restart_rule=1, tolerance=1e-7,
                             max_iterations=200_000)
        assert r.status == "optimal", (k, r.status, r.relative_kkt, r.iterations)
        assert r.relative_kkt < 1e-4
        assert abs(r.objective - o.objective) <= 2e-3 * max(1.0, abs(o.objective)), \
            (k, r.objective, o.objective)


def test_batch_matches_the_single_engine(pkg, engine):
    ps = family(pkg)[:3]
    opt = pkg.PdhgOptions(precision="fp64", max_iterations=100_000, **ADAPTIVE)
    single = []
    for p in ps:
        engine.load(p)
        single.append(engine.solve(opt))
    engine.load_batch(ps)
    for r, s in zip(engine.solve_batch(opt), single):
        assert r.status == s.status == "optimal"
        assert abs(r.iterations - s.iterations) <= 80
        assert abs(r.objective - s.objective) <= 1e-6 * max(1.0, abs(s.objective))
        np.testing.assert_allclose(r.primal, s.primal, rtol=1e-4, atol=1e-5)


def test_invalid_instance_is_reported_and_the_others_solve(pkg, engine):
    ps = family(pkg)[:3]
    bad = dataclasses.replace(ps[1], col_lo=ps[1].col_lo.copy(), col_hi=ps[1].col_hi.copy())
    bad.col_lo[3], bad.col_hi[3] = 2.0, 1.0
    engine.load(bad)
    single = engine.solve(pkg.PdhgOptions(precision="mixed"))
    assert single.status == "numerical_failure"
    engine.load_batch([ps[0], bad, ps[2]])
    rs = engine.solve_batch(pkg.PdhgOptions(precision="mixed", max_iterations=200_000,
                                            **ADAPTIVE))
    assert rs[1].status == "numerical_failure" and rs[1].message == single.message
    assert rs[1].primal.size == 0
    assert rs[0].status == rs[2].status == "optimal"


def test_iteration_limit_with_a_partial_last_period(pkg, engine):
    ps = family(pkg)
    engine.load_batch(ps)
    rs = engine.solve_batch(pkg.PdhgOptions(precision="mixed", max_iterations=130,
                                            tolerance=1e-12, **ADAPTIVE))
    for r in rs:
        assert r.status == "iteration_limit" and r.iterations == 130, (r.status, r.iterations)
        assert r.primal.size > 0


def test_cancel_before_the_first_iteration(pkg, engine):
    ps = family(pkg)[:2]
    engine.load_batch(ps)
    tok = pkg.CancellationToken()
    tok.cancel()
    rs = engine.solve_batch(pkg.PdhgOptions(precision="mixed"), cancel=tok)
    assert all(r.status == "cancelled" and r.iterations == 0 for r in rs)


def test_time_limit_stops_every_instance(pkg, engine):
    ps = [pkg.lpgen.random_equality_lp(300, 800, 6, seed=40 + i) for i in range(3)]
    engine.load_batch(ps)
    rs = engine.solve_batch(pkg.PdhgOptions(precision="fp64", tolerance=1e-15,
                                            max_iterations=50_000_000, time_limit_seconds=0.3,
                                            **ADAPTIVE))
    assert all(r.status == "time_limit" for r in rs), [r.status for r in rs]
    assert all(r.iterations < 50_000_000 for r in rs)


def test_warm_start_from_the_solutions(pkg, engine):
    ps = family(pkg)[:3]
    opt = pkg.PdhgOptions(precision="fp64", max_iterations=100_000, **ADAPTIVE)
    engine.load_batch(ps)
    cold = engine.solve_batch(opt)
    warm = engine.solve_batch(opt, x0=[r.primal for r in cold], y0=[r.dual for r in cold])
    for c, w in zip(cold, warm):
        assert w.status == "optimal" and w.iterations < c.iterations


def test_batch_rejects_exact_mode_and_traces(pkg, engine):
    engine.load_batch(family(pkg)[:2])
    with pytest.raises(pkg.PdhgError):
        engine.solve_batch(pkg.PdhgOptions(precision="fp64_exact"))
    with pytest.raises(pkg.PdhgError):
        engine.solve_batch(pkg.PdhgOptions(precision="mixed", trace_iters=3))


def test_many_uneven_instances(pkg, orc, engine):
    ps = pkg.lpgen.batch_family(48, seed_base=9000, m_lo=20, m_hi=400)
    engine.load_batch(ps)
    rs = engine.solve_batch(pkg.PdhgOptions(precision="mixed", max_iterations=100_000,
                                            **ADAPTIVE))
    assert sum(r.status == "optimal" for r in rs) == len(ps), [r.status for r in rs]
    for k in (0, 17, 47):
        o = orc.oracle_solve(ps[k], termination_rule=1, restart_rule=1, tolerance=1e-7,
                             max_iterations=200_000)
        assert abs(rs[k].objective - o.objective) <= 2e-3 * max(1.0, abs(o.objective))


def test_large_instances_checked_in_parts_match_the_single_engine(pkg, engine):
    # instances of 1,500 x 4,000 and 3,000 x 7,500 (20k and 45k nonzeros): the
    # check sums each in several CTA parts merged by the instance's last part
    ps = [pkg.lpgen.random_equality_lp(1500, 4000, 5, seed=21),
          pkg.lpgen.random_equality_lp(40, 100, 4, seed=23),
          pkg.lpgen.random_equality_lp(3000, 7500, 6, seed=22)]
    opt = pkg.PdhgOptions(precision="fp64", max_iterations=60_000, **ADAPTIVE)
    single = []
    for p in ps:
        engine.load(p)
        single.append(engine.solve(opt))
    engine.load_batch(ps)
    for k, (r, s) in enumerate(zip(engine.solve_batch(opt), single)):
        assert r.status == s.status, (k, r.status, s.status)
        assert abs(r.iterations - s.iterations) <= 80, (k, r.iterations, s.iterations)
        assert abs(r.objective - s.objective) <= 1e-6 * max(1.0, abs(s.objective)), \
            (k, r.objective, s.objective)
