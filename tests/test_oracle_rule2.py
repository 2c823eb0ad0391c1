"""Termination rule 2 (PDLP's relative KKT error) and restart rule 2 in the
oracle, checked against an independent numpy restatement of the measure and
against an LP optimum from scipy's HiGHS.

The reference defines no relative KKT measure (its only rule is the absolute
original-space residual, src/l1/pdhg.cpp:383-389, whose dual part classifies
each bound as active within a tolerance, pdhg.cpp:166-197). Rule 2 is the
engine's extension, restated in oracle/pdhg_oracle.c (pdlp_kkt); these tests
pin that restatement before the GPU tests compare the engine with it.
"""
import numpy as np
import pytest

from conftest import highs_optimum

INF = np.inf


def pdlp_relative_kkt(p, x, y):
    """max(||row violation||_2 / (1 + ||b||_2), ||dual sign violations||_2 /
    (1 + ||c||_2), |p - d| / (1 + |p| + |d|)) at (x, y) in original units and
    sense (y as PdhgResult.dual), b_i the larger finite |row bound|."""
    sgn = -1.0 if p.maximize else 1.0
    A = np.zeros((p.m, p.n))
    for i in range(p.m):
        for k in range(p.row_ptr[i], p.row_ptr[i + 1]):
            A[i, p.col_idx[k]] += p.val[k]
    ax = A @ x
    fl, fu = np.isfinite(p.row_lo), np.isfinite(p.row_hi)
    viol = np.where(fl, np.maximum(p.row_lo - ax, 0), 0) + np.where(fu, np.maximum(ax - p.row_hi, 0), 0)
    b = np.maximum(np.where(fl, np.abs(p.row_lo), 0), np.where(fu, np.abs(p.row_hi), 0))

    def sign_viol(v, lo, hi):
        l, h = np.isfinite(lo), np.isfinite(hi)
        out = np.where(l & h, 0.0, np.where(l, np.maximum(-v, 0), np.where(h, np.maximum(v, 0), np.abs(v))))
        return out

    def clipped(v, lo, hi):
        lo0 = np.where(np.isfinite(lo), lo, 0.0)
        hi0 = np.where(np.isfinite(hi), hi, 0.0)
        return np.where(v > 0, v * lo0, np.where(v < 0, v * hi0, 0.0))

    y_int = sgn * y
    r_int = sgn * (p.c - A.T @ y)
    d = np.concatenate([sign_viol(y_int, p.row_lo, p.row_hi), sign_viol(r_int, p.col_lo, p.col_hi)])
    pobj = sgn * (p.c @ x + p.obj_const)
    dobj = sgn * p.obj_const + clipped(y_int, p.row_lo, p.row_hi).sum() + clipped(r_int, p.col_lo, p.col_hi).sum()
    parts = (np.linalg.norm(viol) / (1 + np.linalg.norm(b)),
             np.linalg.norm(d) / (1 + np.linalg.norm(p.c)),
             abs(pobj - dobj) / (1 + abs(pobj) + abs(dobj)))
    return max(parts)


def cases(pkg):
    L = pkg.lpgen
    return {"equality_60x150": L.random_equality_lp(60, 150, 4, seed=11),
            "transportation_20x50": L.transportation_lp(20, 50, seed=1000),
            "badly_scaled_120x300": L.badly_scaled_lp(120, 300, 5, seed=2000),
            "maximize_40x90": L.random_equality_lp(40, 90, 4, seed=12, maximize=True)}


@pytest.mark.parametrize("name", ["equality_60x150", "transportation_20x50",
                                  "badly_scaled_120x300", "maximize_40x90"])
@pytest.mark.parametrize("restart_rule,pw", [(1, 0), (2, 0), (2, 1)])
def test_rule2_solutions_meet_the_measure_and_the_optimum(pkg, orc, name, restart_rule, pw):
    p = cases(pkg)[name]
    r = orc.oracle_solve(p, tolerance=1e-4, termination_rule=2, restart_rule=restart_rule,
                         primal_weight_update=pw, max_iterations=400_000)
    assert r.status == "optimal", (r.status, r.iterations, r.relative_kkt)
    assert r.relative_kkt < 1e-4
    # the reported value is the measure at the returned point
    assert pdlp_relative_kkt(p, r.primal, r.dual) == pytest.approx(r.relative_kkt, rel=1e-9, abs=1e-14)
    # 1e-4 relative KKT (its gap part relative to 1 + |p| + |d|) puts the
    # objective within a few 1e-4 of the optimum
    opt = highs_optimum(p)
    assert abs(r.objective - opt) <= 5e-4 * (1 + abs(opt)), (r.objective, opt)


def test_rule2_reaches_the_tolerance_before_the_max_norm_rule(pkg, orc):
    # the max-norm rule's dual part only drops once every bound is classified
    # exactly (active within the tolerance); rule 2 measures distances
    p = pkg.lpgen.transportation_lp(40, 100, seed=1000)
    r1 = orc.oracle_solve(p, termination_rule=1, restart_rule=1, max_iterations=200_000)
    r2 = orc.oracle_solve(p, termination_rule=2, restart_rule=2, max_iterations=200_000)
    assert r1.status == r2.status == "optimal"
    assert r2.iterations < r1.iterations


def test_restart_rule_2_restarts_on_its_measure(pkg, orc):
    # restart rule 2 measures average and current by rule 2's parts; on an
    # equality LP it restarts and still converges
    p = pkg.lpgen.random_equality_lp(30, 70, 3, seed=5)
    r = orc.oracle_solve(p, termination_rule=2, restart_rule=2, max_iterations=100_000)
    assert r.status == "optimal" and r.restarts >= 1


@pytest.mark.parametrize("name", ["equality_60x150", "transportation_20x50",
                                  "badly_scaled_120x300", "maximize_40x90"])
@pytest.mark.parametrize("pw", [0, 1])
def test_halpern_solutions_meet_the_measure_and_the_optimum(pkg, orc, name, pw):
    # the reflected restarted Halpern iteration (option halpern) on rule 2
    p = cases(pkg)[name]
    r = orc.oracle_solve(p, tolerance=1e-4, termination_rule=2, restart_rule=2,
                         primal_weight_update=pw, halpern=1, max_iterations=400_000)
    assert r.status == "optimal", (r.status, r.iterations, r.relative_kkt)
    assert r.relative_kkt < 1e-4
    assert pdlp_relative_kkt(p, r.primal, r.dual) == pytest.approx(r.relative_kkt, rel=1e-9, abs=1e-14)
    # the reported point is T(z): inside the column bounds
    assert np.all(r.primal >= p.col_lo - 1e-12) and np.all(r.primal <= p.col_hi + 1e-12)
    opt = highs_optimum(p)
    assert abs(r.objective - opt) <= 5e-4 * (1 + abs(opt)), (r.objective, opt)


def test_halpern_takes_fewer_iterations_than_the_average(pkg, orc):
    L = pkg.lpgen
    for p, pw in ((L.transportation_lp(100, 250, seed=1000), 0),
                  (L.random_equality_lp(400, 1000, 5, seed=0), 1)):
        kw = dict(tolerance=1e-4, termination_rule=2, restart_rule=2, primal_weight_update=pw,
                  max_iterations=200_000)
        avg = orc.oracle_solve(p, **kw)
        hal = orc.oracle_solve(p, halpern=1, **kw)
        assert avg.status == hal.status == "optimal"
        assert hal.iterations < avg.iterations, (hal.iterations, avg.iterations)
