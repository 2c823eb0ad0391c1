"""The no-allocation SpMV entry point (pdhg_csr_spmv_noalloc) through the C-ABI.

It serves callers that cannot allocate device memory when they need the
product (frameworks with their own memory pool, allocation-free real-time
loops). The test owns every device
buffer (made with torch), calls the entry point on torch's current stream and
requires results bit-identical to the allocating pdhg_csr_spmv, on consecutive
calls with different shapes (the shared scratch keeps the previous call's
contents and must be cleared by each call). This file is named to be collected
last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PDHG_ERR_INVALID_ARGUMENT = 3


def _entry(pkg):
    f = pkg.pdhg.lib().pdhg_csr_spmv_noalloc
    f.argtypes = [C.c_int, C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _call(pkg, p, transpose, alpha, x, beta, y0):
    import torch
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    rp, ci, va, dx, dy = t(p.row_ptr), t(p.col_idx), t(p.val), t(x), t(y0)
    stream = torch.cuda.current_stream(dev)
    rc = _entry(pkg)(int(transpose), p.m, p.n, p.nnz, rp.data_ptr(), ci.data_ptr(),
                     va.data_ptr(), alpha, dx.data_ptr(), beta, dy.data_ptr(),
                     stream.cuda_stream)
    assert rc == 0, rc
    stream.synchronize()
    return dy.cpu().numpy()


def test_noalloc_spmv_matches_the_allocating_entry_point(pkg):
    cases = [pkg.lpgen.badly_scaled_lp(300, 800, 5, seed=41),
             pkg.lpgen.random_equality_lp(1200, 5000, 7, seed=42),
             pkg.lpgen.badly_scaled_lp(300, 800, 5, seed=41)]
    for i, p in enumerate(cases):  # consecutive calls, different shapes, then a repeat
        rng = np.random.default_rng(i)
        x_t = rng.standard_normal(p.m)
        y_t = rng.standard_normal(p.n)
        expected = pkg.csr_spmv(p, -0.75, x_t, 1.5, y_t, transpose=True)
        assert np.array_equal(_call(pkg, p, True, -0.75, x_t, 1.5, y_t), expected), i
        expected = pkg.csr_spmv(p, 0.5, x_t, 0.0, np.zeros(p.n), transpose=True)
        assert np.array_equal(_call(pkg, p, True, 0.5, x_t, 0.0, np.full(p.n, np.nan)),
                              expected), i
        x = rng.standard_normal(p.n)
        y = rng.standard_normal(p.m)
        expected = pkg.csr_spmv(p, 2.0, x, -1.0, y)
        assert np.array_equal(_call(pkg, p, False, 2.0, x, -1.0, y), expected), i


def test_noalloc_spmv_refuses_sizes_beyond_its_scratch(pkg):
    f = _entry(pkg)
    rp = np.zeros(2, dtype=np.int32)
    # 300,000 columns exceed the 262,144 the fixed scratch holds; refused before any work
    rc = f(1, 1, 300_000, 0, rp.ctypes.data, None, None, 1.0, None, 0.0, rp.ctypes.data, None)
    assert rc == PDHG_ERR_INVALID_ARGUMENT
    rc = f(1, 10, 100, 300_000, rp.ctypes.data, rp.ctypes.data, rp.ctypes.data, 1.0,
           rp.ctypes.data, 0.0, rp.ctypes.data, None)
    assert rc == PDHG_ERR_INVALID_ARGUMENT
