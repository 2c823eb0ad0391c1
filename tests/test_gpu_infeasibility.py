"""Infeasibility detection (engine extension, option infeasibility_detection).

At every check the change of y since the previous check, in original units, is
tested as a sov::FarkasCertificate (src/l1/duals.cpp:36-79). A primal
infeasible LP must stop with status "primal_infeasible" and a certificate that
the reference's own checker accepts (or, without the reference sources, the
oracle's restatement of it, pinned to the reference on the CPU); a feasible LP
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
    assert r.farkas is not None and r.farkas.shape == (p.m,)
    assert np.max(np.abs(r.farkas)) == pytest.approx(1.0)
    ok, ranges = certifies(orc, p, r.farkas)
    assert ok, (ranges, r.message)
    # the same LP without the detection runs to its limit, like the reference
    r0 = engine.solve(pkg.PdhgOptions(precision=precision, **dict(KW, max_iterations=2000)))
    assert r0.status == "iteration_limit"


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_detection_leaves_a_feasible_solve_unchanged(pkg, engine, precision):
    p = pkg.lpgen.random_equality_lp(200, 500, 5, seed=41)
    engine.load(p)
    off = engine.solve(pkg.PdhgOptions(precision=precision, **KW))
    on = engine.solve(pkg.PdhgOptions(precision=precision, infeasibility_detection=True, **KW))
    assert off.status == on.status == "optimal"
    assert (off.iterations, off.restarts, off.objective) == (on.iterations, on.restarts, on.objective)
    assert np.array_equal(off.primal, on.primal) and np.array_equal(off.dual, on.dual)
    assert on.farkas is None


def test_exact_mode_and_batches_refuse_the_detection(pkg, engine):
    p = pkg.lpgen.random_equality_lp(30, 70, 3, seed=5)
    engine.load(p)
    with pytest.raises(pkg.pdhg.PdhgError):
        engine.solve(pkg.PdhgOptions(infeasibility_detection=True))
    engine.load_batch([p, p])
    with pytest.raises(pkg.pdhg.PdhgError):
        engine.solve_batch(pkg.PdhgOptions(precision="mixed", infeasibility_detection=True))
