"""The oracle against the golden fixtures (reference outputs committed in
tests/golden/), and the hand-derived answers of the reference's own tests.

Runs everywhere (no reference sources needed): this is what pins the oracle
on the GPU box, where the oracle then checks the CUDA engine.
"""
import hashlib

import numpy as np
import pytest

from conftest import PDHG_CASES, golden_problem, load_golden

FAST = [c for c in PDHG_CASES if not c.startswith("c0_")]


def check_against_golden(res, g, exact=True):
    assert res.status == g["ref_status"], (res.status, g["ref_status"], res.message)
    assert res.message == g["ref_message"]
    assert res.iterations == g["ref_iterations"]
    assert res.restarts == g["ref_restarts"]
    for f in ("objective", "primal_infeasibility", "dual_infeasibility", "duality_gap",
              "operator_norm_estimate"):
        assert getattr(res, f) == g["ref_" + f], f
    if g["ref_has_point"]:
        for f in ("primal", "dual", "reduced_costs"):
            assert np.array_equal(getattr(res, f), g["ref_" + f]), f


@pytest.mark.parametrize("name", FAST)
def test_oracle_reproduces_reference_fixture(pkg, orc, name):
    g = load_golden(name)
    p = golden_problem(pkg, g)
    tr = 100 if "trace_x" in g else 0
    r = orc.oracle_solve(p, trace_iters=tr, **g["options"])
    check_against_golden(r, g)
    if tr:
        assert np.array_equal(r.trace_x, g["trace_x"])
        assert np.array_equal(r.trace_y, g["trace_y"])


def trace_digests(trace):
    """SHA-256 of each traced iterate's FP64 bytes (as make_golden.py stores them)."""
    return np.stack([np.frombuffer(hashlib.sha256(np.ascontiguousarray(row).tobytes()).digest(),
                                   dtype=np.uint8) for row in trace])


def test_oracle_reproduces_the_2000x5000_fixture(pkg, orc):
    g = load_golden("c0_2000x5000_tol1e-4")
    p = golden_problem(pkg, g)
    r = orc.oracle_solve(p, trace_iters=100, **g["options"])
    check_against_golden(r, g)
    keep = g["trace_iters_kept"]
    assert np.array_equal(r.trace_x[keep], g["trace_x"])
    assert np.array_equal(r.trace_y[keep], g["trace_y"])
    assert np.array_equal(trace_digests(r.trace_x), g["trace_digest_x"])
    assert np.array_equal(trace_digests(r.trace_y), g["trace_digest_y"])


def test_oracle_reproduces_the_first_100_iterates_at_tol_1e6(pkg, orc):
    # the stated tolerance of the 2,000 x 5,000 LP: the reference ends
    # iteration_limit at its 1,000,000-iteration cap (about 2 minutes of CPU
    # here, so only the first 100 iterates are checked on the CPU; the GPU
    # tests compare the engine's whole run with the fixture)
    g = load_golden("c0_2000x5000_tol1e-6")
    assert g["ref_status"] == "iteration_limit" and g["ref_iterations"] == 1_000_000
    p = golden_problem(pkg, g)
    r = orc.oracle_solve(p, trace_iters=100, max_iterations=100, **g["options"])
    assert np.array_equal(trace_digests(r.trace_x), g["trace_digest_x"])
    assert np.array_equal(trace_digests(r.trace_y), g["trace_digest_y"])
    keep = g["trace_iters_kept"]
    assert np.array_equal(r.trace_x[keep], g["trace_x"])
    assert np.array_equal(r.trace_y[keep], g["trace_y"])


# Hand-derived optima of tests/test_pdhg.cpp (checked there to 5e-4).
HAND = {
    "pdhg_two_variable_optimum_matches_simplex": (10.0 / 3.0, {0: 8 / 3, 1: 2 / 3}),
    "pdhg_minimize_with_a_binding_lower_bound": (8.0, {0: 0.0, 1: 4.0}),
    "pdhg_equality_row": (10.0, {}),
    "pdhg_column_bound_forces_the_optimum": (-3.0, {0: 3.0}),
    "pdhg_agrees_with_a_hand_verified_degenerate_optimum": (-4.0, {}),
    "smoke_tiny_lp": (-10.0 / 3.0, {0: 8 / 3, 1: 2 / 3}),
}


@pytest.mark.parametrize("name", sorted(HAND))
def test_fixture_meets_the_hand_derived_optimum(name):
    g = load_golden(name)
    obj, xs = HAND[name]
    assert g["ref_status"] == "optimal"
    assert abs(g["ref_objective"] - obj) < 5e-4
    for j, v in xs.items():
        assert abs(g["ref_primal"][j] - v) < 1e-3


def test_time_limit_fixture_reports_a_point():
    g = load_golden("pdhg_a_time_limit_before_the_first_restart_check_still_reports_a_point")
    assert g["ref_status"] == "time_limit" and g["ref_iterations"] == 0
    assert g["ref_primal"].shape == (2,)


def test_backend_known_answers(pkg, orc):
    g = load_golden("backend_known_answers")
    A = golden_problem(pkg, g)
    assert np.array_equal(g["ax"], [-1.0, 18.0, 1.0, 15.0])
    assert np.array_equal(g["aty"], [5.0, 6.0, 27.0])
    assert np.array_equal(g["ax_alpha_beta"], [1.0, 39.0, 5.0, 33.0])
    assert np.array_equal(orc.oracle_spmv(A, 1.0, g["x"], 0.0, np.zeros(4)), g["ax"])
    assert np.array_equal(orc.oracle_spmv(A, 2.0, g["x"], 3.0, np.ones(4)), g["ax_alpha_beta"])
    assert np.array_equal(orc.oracle_spmv(A, 1.0, g["y"], 0.0, np.zeros(3), transpose=True), g["aty"])
    assert not np.isnan(orc.oracle_spmv(A, 1.0, g["x"], 0.0, np.full(4, np.nan))).any()


def test_scaling_fixture(pkg, orc):
    g = load_golden("scaling_ill_scaled")
    S = golden_problem(pkg, g)
    rs, cs = orc.oracle_scaling(S)
    assert np.array_equal(rs, g["row_scale"]) and np.array_equal(cs, g["col_scale"])
    rs, cs = orc.oracle_scaling(S, apply_pock_chambolle=0)
    assert np.array_equal(rs, g["row_scale_ruiz"]) and np.array_equal(cs, g["col_scale_ruiz"])
