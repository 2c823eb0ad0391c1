"""Infeasibility detection (engine extension, option infeasibility_detection).

At every check the change of y since the previous check, in original units, is
tested as a sov::FarkasCertificate (src/l1/duals.cpp:36-79), and the change of
x as a ray of unbounded descent. A primal infeasible LP must stop with status
"primal_infeasible" and a certificate that the reference's own checker accepts
(or, without the reference sources, the oracle's restatement of it, pinned to
the reference on the CPU); an unbounded LP must stop with status
"dual_infeasible" and a ray that the oracle's ray test accepts; a feasible LP
must solve exactly as with the detection off; fp64_exact (the reference's
behaviour) and the batched engine refuse the option.
"""
import numpy as np
import pytest

from conftest import golden_problem, load_golden

pytestmark = pytest.mark.gpu

KW = dict(termination_rule="relative_kkt", restart_rule="adaptive", max_iterations=40_000)


@pytest.fixture(scope="module")
def engine(pkg):
    e = pkg.Engine(0)
    yield e
    e.close()


def certifies(orc, p, y):
    check = orc.reference_certifies if orc.ref_available() else orc.oracle_certifies
    ok, ranges = check(p, y, 1e-6)
    return ok, ranges


def with_rows(p, rows):
    """p with dense rows appended: [(coefficients (n), lo, hi), ...]."""
    rp, ci, val = list(p.row_ptr), list(p.col_idx), list(p.val)
    lo, hi = list(p.row_lo), list(p.row_hi)
    for coef, rlo, rhi in rows:
        nz = np.flatnonzero(coef)
        ci += list(nz)
        val += list(coef[nz])
        rp.append(rp[-1] + len(nz))
        lo.append(rlo)
        hi.append(rhi)
    return p.__class__(m=p.m + len(rows), n=p.n, row_ptr=rp, col_idx=ci, val=val, c=p.c,
                       col_lo=p.col_lo, col_hi=p.col_hi, row_lo=lo, row_hi=hi,
                       obj_const=p.obj_const, maximize=p.maximize, name=p.name + "_infeasible")


def with_block(p, c, lo, hi, rows):
    """p with new columns (costs c, bounds lo, hi) and new rows over those
    columns only, [(coefficients over the new columns, lo, hi), ...]: a block
    beside p's own."""
    rp, ci, val = list(p.row_ptr), list(p.col_idx), list(p.val)
    rlo, rhi = list(p.row_lo), list(p.row_hi)
    for coef, a, b in rows:
        coef = np.asarray(coef, dtype=np.float64)
        nz = np.flatnonzero(coef)
        ci += list(p.n + nz)
        val += list(coef[nz])
        rp.append(rp[-1] + len(nz))
        rlo.append(a)
        rhi.append(b)
    return p.__class__(m=p.m + len(rows), n=p.n + len(c), row_ptr=rp, col_idx=ci, val=val,
                       c=np.r_[p.c, c], col_lo=np.r_[p.col_lo, lo], col_hi=np.r_[p.col_hi, hi],
                       row_lo=rlo, row_hi=rhi, obj_const=p.obj_const, maximize=p.maximize,
                       name=p.name + "_unbounded")


def unbounded_family(pkg):
    base = pkg.lpgen.random_equality_lp(200, 500, 5, seed=41)
    inf = np.inf
    # x_a - x_b = 0, x_a, x_b >= 0, cost -x_a + x_b / 2: falls by 1/2 along (1, 1)
    pair = with_block(base, [-1.0, 0.5], [0.0, 0.0], [inf, inf], [([1.0, -1.0], 0.0, 0.0)])
    # a free column of cost 1 with only x_f <= 5: falls along -1
    free = with_block(base, [1.0], [-inf], [inf], [([1.0], -inf, 5.0)])
    # min -x1 with x1 - x2 <= 5, x >= 0; and max x1 over the same rows
    tiny = golden_problem(pkg, load_golden("smoke_tiny_unbounded"))
    tiny_max = golden_problem(pkg, load_golden("smoke_tiny_unbounded"))
    tiny_max.c, tiny_max.maximize = np.array([1.0, 0.0]), True
    # the reference's two fixtures with every bound type: HiGHS (scipy) finds
    # both unbounded with a feasible primal; the reference runs to its limit
    mb = golden_problem(pkg, load_golden("mixed_bounds_50x90"))
    mb7 = golden_problem(pkg, load_golden("mixed_bounds_period7"))
    return {"tiny": tiny, "tiny_max": tiny_max, "pair": pair, "free": free,
            "mixed_bounds": mb, "mixed_bounds_period7": mb7}


def infeasible_family(pkg):
    base = pkg.lpgen.random_equality_lp(200, 500, 5, seed=41)
    n = base.n
    # the box 0 <= x <= 10 caps sum x at 10 n
    over_box = with_rows(base, [(np.ones(n), 10.0 * n + 100.0, np.inf)])
    rng = np.random.default_rng(42)
    a = rng.standard_normal(n) * (rng.random(n) < 0.1)
    # the same combination asked to be <= 1 and >= 3
    contradictory = with_rows(base, [(a, -np.inf, 1.0), (a, 3.0, np.inf)])
    tiny = golden_problem(pkg, load_golden("smoke_tiny_infeasible"))
    return {"tiny": tiny, "over_box": over_box, "contradictory": contradictory}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["tiny", "over_box", "contradictory"])
def test_infeasible_lps_stop_with_a_certificate(pkg, orc, engine, precision, name):
    p = infeasible_family(pkg)[name]
    engine.load(p)
    r = engine.solve(pkg.PdhgOptions(precision=precision, infeasibility_detection=True, **KW))
    assert r.status == "primal_infeasible", (r.status, r.iterations, r.message)
    assert r.farkas is not None and r.farkas.shape == (p.m,) and r.ray is None
    assert np.max(np.abs(r.farkas)) == pytest.approx(1.0)
    ok, ranges = certifies(orc, p, r.farkas)
    assert ok, (ranges, r.message)
    # the same LP without the detection runs to its limit, like the reference
    r0 = engine.solve(pkg.PdhgOptions(precision=precision, **dict(KW, max_iterations=2000)))
    assert r0.status == "iteration_limit"


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["tiny", "tiny_max", "pair", "free", "mixed_bounds",
                                  "mixed_bounds_period7"])
def test_unbounded_lps_stop_with_a_ray(pkg, orc, engine, precision, name):
    p = unbounded_family(pkg)[name]
    engine.load(p)
    r = engine.solve(pkg.PdhgOptions(precision=precision, infeasibility_detection=True,
                                     **dict(KW, max_iterations=200_000)))
    assert r.status == "dual_infeasible", (r.status, r.iterations, r.message)
    assert r.ray is not None and r.ray.shape == (p.n,) and r.farkas is None
    assert np.max(np.abs(r.ray)) == pytest.approx(1.0)
    ok, obj, viol = orc.ray_certifies(p, r.ray)
    assert ok, (obj, viol, r.message)
    r0 = engine.solve(pkg.PdhgOptions(precision=precision, **dict(KW, max_iterations=2000)))
    assert r0.status == "iteration_limit"


def feasible_family(pkg):
    # boxed columns; columns with only a lower end (x >= 0); every row type
    # with the one-sided columns of mixed_bounds_50x90 boxed at 100 from their
    # finite end (HiGHS: optimal, -1023.55)
    mb = golden_problem(pkg, load_golden("mixed_bounds_50x90"))
    lo, hi = mb.col_lo.copy(), mb.col_hi.copy()
    lo_only, hi_only = np.isfinite(lo) & ~np.isfinite(hi), ~np.isfinite(lo) & np.isfinite(hi)
    hi[lo_only] = lo[lo_only] + 100.0
    lo[hi_only] = hi[hi_only] - 100.0
    mb.col_lo, mb.col_hi = lo, hi
    return {"boxed": pkg.lpgen.random_equality_lp(200, 500, 5, seed=41),
            "transportation": pkg.lpgen.transportation_lp(30, 60, seed=7),
            "mixed_boxed": mb}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["boxed", "transportation", "mixed_boxed"])
def test_detection_leaves_a_feasible_solve_unchanged(pkg, engine, precision, name):
    p = feasible_family(pkg)[name]
    engine.load(p)
    off = engine.solve(pkg.PdhgOptions(precision=precision, **KW))
    on = engine.solve(pkg.PdhgOptions(precision=precision, infeasibility_detection=True, **KW))
    assert off.status == on.status == "optimal"
    assert (off.iterations, off.restarts, off.objective) == (on.iterations, on.restarts, on.objective)
    assert np.array_equal(off.primal, on.primal) and np.array_equal(off.dual, on.dual)
    assert on.farkas is None and on.ray is None


def test_exact_mode_and_batches_refuse_the_detection(pkg, engine):
    p = pkg.lpgen.random_equality_lp(30, 70, 3, seed=5)
    engine.load(p)
    with pytest.raises(pkg.pdhg.PdhgError):
        engine.solve(pkg.PdhgOptions(infeasibility_detection=True))
    engine.load_batch([p, p])
    with pytest.raises(pkg.pdhg.PdhgError):
        engine.solve_batch(pkg.PdhgOptions(precision="mixed", infeasibility_detection=True))
