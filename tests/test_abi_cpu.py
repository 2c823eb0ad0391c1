"""The C-ABI library without a GPU: it loads, exports exactly what
include/pdhg_b200.h declares, and its host-side entry points (defaults,
strings, scaling) agree with the reference. No compute call needs a device here.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_problem, load_golden

HEADER = os.path.join(ROOT, "include", "pdhg_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:int|void\*?|const char\*)\s+(pdhg_\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.pdhg.lib()
    names = declared_functions()
    assert "pdhg_solve" in names and "pdhg_load_problem" in names
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.pdhg.LIB_PATH],
                         capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (pdhg_\w+)", out))
    assert set(names) <= exported


def test_defaults_are_the_reference_defaults(pkg):
    lib = pkg.pdhg.lib()
    o = pkg.pdhg._Options()
    lib.pdhg_default_options(C.byref(o))
    # include/sovereign/pdhg.hpp:89-117, scaling.hpp:299-309
    assert o.tolerance == 1e-4 and o.max_iterations == 1_000_000
    assert o.time_limit_seconds == 0.0 and o.restart_check_period == 40
    assert o.restart_sufficient_decrease == 0.5 and o.step_size_safety == 0.9
    assert o.power_iterations == 30 and o.verbose == 0
    assert o.ruiz_iterations == 8 and o.ruiz_tolerance == 1e-2
    assert o.pock_chambolle_alpha == 1.0 and o.apply_ruiz == 1 and o.apply_pock_chambolle == 1
    assert o.precision == 0 and o.termination_rule == 0
    assert o.autotune == 1  # an engine extension; it never applies to fp64_exact
    assert o.infeasibility_detection == 0  # extension, off: the reference never reports it
    assert o.halpern == 0  # extension, off: the reference's averaged PDHG
    assert lib.pdhg_abi_version() == 4
    d = pkg.PdhgOptions()
    assert d.tolerance == o.tolerance and d.max_iterations == o.max_iterations


def test_status_and_error_strings(pkg):
    lib = pkg.pdhg.lib()
    assert [lib.pdhg_status_string(i).decode() for i in range(6)] == [
        "optimal", "iteration_limit", "time_limit", "numerical_failure", "not_solved",
        "cancelled"]
    assert lib.pdhg_status_string(6).decode() == "primal_infeasible"  # engine extension
    assert lib.pdhg_status_string(7).decode() == "dual_infeasible"  # engine extension
    assert lib.pdhg_error_string(3).decode() == "invalid argument"
    assert lib.pdhg_error_string(6).decode() == "backend error"


def test_engine_scaling_is_the_reference_scaling(pkg, orc):
    g = load_golden("scaling_ill_scaled")
    S = golden_problem(pkg, g)
    rs, cs = pkg.scaling(S)
    assert np.array_equal(rs, g["row_scale"]) and np.array_equal(cs, g["col_scale"])
    rs, cs = pkg.scaling(S, pkg.PdhgOptions(apply_pock_chambolle=False))
    assert np.array_equal(rs, g["row_scale_ruiz"]) and np.array_equal(cs, g["col_scale_ruiz"])
    p = pkg.lpgen.badly_scaled_lp(400, 900, 6, seed=3)
    a, b = pkg.scaling(p), orc.oracle_scaling(p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_no_cpu_fallback_without_a_device(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = pkg.lpgen.random_equality_lp(10, 20, 2, seed=0)
    with pytest.raises(pkg.PdhgError):
        pkg.Pdhg().solve(p)
    with pytest.raises(pkg.PdhgError):
        pkg.csr_spmv(p, 1.0, np.ones(20), 0.0, np.zeros(10))


def test_header_documents_each_entry_with_a_reference_citation():
    src = open(HEADER).read()
    for n in declared_functions():
        i = src.index(n + "(")
        end = src.rfind("*/", 0, i)
        semi = src.index(";", i)
        block = src[src.rfind("/*", 0, end): i] + src[i: src.index("\n", semi)]
        assert re.search(r"\w+\.(?:cpp|hpp):\d+", block) or n in (
            "pdhg_abi_version", "pdhg_default_options", "pdhg_last_error",
            "pdhg_profile_kernels", "pdhg_destroy", "pdhg_stream",
            "pdhg_csr_spmv_noalloc", "pdhg_get_tuning", "pdhg_get_batch_tuning",
            "pdhg_gemm_bf16") or \
            n.startswith("pdhg_mlp_"), n  # the warm start's network: no reference counterpart


def test_results_hand_over_the_written_point_and_nothing_else(pkg):
    # the result owns views of the buffers the engine wrote (no second copy of
    # a 10M-column point); without want_point the engine wrote nothing and the
    # point fields stay empty, whatever has_point says
    P = pkg.pdhg
    info = P._Info()
    info.status = P.STATUS.index("iteration_limit")
    info.has_point = 1
    x, y, rc = np.arange(6.0), np.arange(3.0), -np.arange(6.0)
    r = P._result(info, x[:5], y[:2], rc[:5])
    assert r.primal.base is x and r.dual.base is y and r.reduced_costs.base is rc
    assert np.array_equal(r.primal, x[:5]) and r.farkas is None and r.ray is None
    r = P._result(info, x[:5], y[:2], rc[:5], want_point=False)
    assert r.primal.size == r.dual.size == r.reduced_costs.size == 0
    info.status = P.STATUS.index("primal_infeasible")
    info.has_point = 0
    assert np.array_equal(P._result(info, x, y, rc).farkas, y)
    assert P._result(info, x, y, rc, want_point=False).farkas is None
    info.status = P.STATUS.index("dual_infeasible")
    assert np.array_equal(P._result(info, x, y, rc).ray, x)
    assert P._result(info, x, y, rc, want_point=False).ray is None
