"""The no-allocation SpMV entry point (pdhg_csr_spmv_noalloc) through the C-ABI.

It serves callers that cannot allocate device memory when they need the
product (frameworks with their own memory pool, allocation-free real-time
loops). The test owns every device buffer (made with torch), calls the entry
point on torch's current stream and requires results bit-identical to the
allocating pdhg_csr_spmv and to the oracle's restatement of the reference's
Backend::spmv / spmv_transpose, on consecutive calls with different shapes
(the shared scratch keeps the previous call's contents and must be cleared by
each call), at the scratch's size limits, on empty shapes, with duplicate
entries, and on malformed CSR input, which must come back as NaN in every
output entry. This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PDHG_ERR_INVALID_ARGUMENT = 3
LIMIT = 262_144  # columns and nonzeros the fixed scratch holds (transposed products)


def _entry(pkg):
    f = pkg.pdhg.lib().pdhg_csr_spmv_noalloc
    f.argtypes = [C.c_int, C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _call(pkg, p, transpose, alpha, x, beta, y0, nnz=None):
    import torch
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    rp, ci, va, dx, dy = (t(p.row_ptr.astype(np.int32)), t(p.col_idx.astype(np.int32)),
                          t(p.val), t(x), t(y0))
    ptr = lambda a: a.data_ptr() if a.numel() else None  # noqa: E731
    stream = torch.cuda.current_stream(dev)
    rc = _entry(pkg)(int(transpose), p.m, p.n, p.nnz if nnz is None else nnz, rp.data_ptr(),
                     ptr(ci), ptr(va), alpha, ptr(dx), beta, ptr(dy), stream.cuda_stream)
    assert rc == 0, rc
    stream.synchronize()
    return dy.cpu().numpy()


def _both_ways(pkg, orc, p, seed):
    """Transposed (beta != 0 and beta == 0 on a NaN-filled y) and plain
    products: the no-allocation entry point against the allocating one and
    the oracle."""
    rng = np.random.default_rng(seed)
    x_t = rng.standard_normal(p.m)
    y_t = rng.standard_normal(p.n)
    got = _call(pkg, p, True, -0.75, x_t, 1.5, y_t)
    assert np.array_equal(got, pkg.csr_spmv(p, -0.75, x_t, 1.5, y_t, transpose=True))
    assert np.array_equal(got, orc.oracle_spmv(p, -0.75, x_t, 1.5, y_t, transpose=True))
    got = _call(pkg, p, True, 0.5, x_t, 0.0, np.full(p.n, np.nan))
    assert np.array_equal(got, pkg.csr_spmv(p, 0.5, x_t, 0.0, np.zeros(p.n), transpose=True))
    assert np.array_equal(got, orc.oracle_spmv(p, 0.5, x_t, 0.0, np.zeros(p.n), transpose=True))
    x = rng.standard_normal(p.n)
    y = rng.standard_normal(p.m)
    got = _call(pkg, p, False, 2.0, x, -1.0, y)
    assert np.array_equal(got, pkg.csr_spmv(p, 2.0, x, -1.0, y))
    assert np.array_equal(got, orc.oracle_spmv(p, 2.0, x, -1.0, y))


def _csr(pkg, m, n, rows_cols, rng):
    """Problem with the given per-row column lists (kept in order, duplicates
    allowed) and N(0,1) values."""
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum([len(c) for c in rows_cols], out=row_ptr[1:])
    col_idx = (np.concatenate(rows_cols) if rows_cols else np.zeros(0)).astype(np.int64)
    z = np.zeros
    return pkg.Problem(m=m, n=n, row_ptr=row_ptr, col_idx=col_idx,
                       val=rng.standard_normal(col_idx.size), c=z(n), col_lo=z(n), col_hi=z(n),
                       row_lo=z(m), row_hi=z(m), name="noalloc_case")


def test_noalloc_spmv_matches_the_allocating_entry_point_and_the_oracle(pkg, orc):
    cases = [pkg.lpgen.badly_scaled_lp(300, 800, 5, seed=41),
             pkg.lpgen.random_equality_lp(1200, 5000, 7, seed=42),
             pkg.lpgen.badly_scaled_lp(300, 800, 5, seed=41)]
    for i, p in enumerate(cases):  # consecutive calls, different shapes, then a repeat
        _both_ways(pkg, orc, p, i)


def test_noalloc_spmv_at_the_scratch_limits(pkg, orc):
    rng = np.random.default_rng(7)
    # 2,048 rows of 128 distinct columns each: n and nnz both at 262,144
    rows = [np.sort(rng.choice(LIMIT, size=128, replace=False)) for _ in range(2048)]
    p = _csr(pkg, 2048, LIMIT, rows, rng)
    assert p.nnz == LIMIT and p.n == LIMIT
    _both_ways(pkg, orc, p, 1)
    # a row longer than a warp's worth and a column holding most rows
    rows = [np.concatenate([[0], np.sort(rng.choice(np.arange(1, 5000), size=k, replace=False))])
            for k in rng.integers(0, 400, size=700)]
    _both_ways(pkg, orc, _csr(pkg, 700, 5000, rows, rng), 2)


def test_noalloc_spmv_on_empty_shapes(pkg, orc):
    rng = np.random.default_rng(3)
    for m, n in ((0, 5), (5, 0), (0, 0), (4, 6)):
        rows = [np.zeros(0, dtype=np.int64) for _ in range(m)]
        p = _csr(pkg, m, n, rows, rng)
        x_t, y_t = rng.standard_normal(m), rng.standard_normal(n)
        assert np.array_equal(_call(pkg, p, True, 1.0, x_t, 2.0, y_t), 2.0 * y_t)
        x, y = rng.standard_normal(n), rng.standard_normal(m)
        assert np.array_equal(_call(pkg, p, False, 1.0, x, 0.0, np.full(m, np.nan)), np.zeros(m))


def test_noalloc_spmv_keeps_duplicates_in_their_order(pkg, orc):
    rng = np.random.default_rng(5)
    rows = []
    for _ in range(400):
        c = rng.integers(0, 300, size=int(rng.integers(0, 40)))
        rows.append(np.concatenate([c, c[: len(c) // 2]]))  # repeated (row, column) pairs
    p = _csr(pkg, 400, 300, rows, rng)
    p.val = np.exp(rng.uniform(-20, 20, p.nnz)) * rng.choice([-1.0, 1.0], p.nnz)  # order-sensitive
    _both_ways(pkg, orc, p, 3)


def test_noalloc_spmv_turns_a_malformed_csr_into_nan(pkg):
    rng = np.random.default_rng(9)
    good = _csr(pkg, 6, 10, [np.arange(k) for k in (1, 3, 0, 2, 4, 2)], rng)
    x_t, y_t = rng.standard_normal(6), rng.standard_normal(10)
    bad_col = _csr(pkg, 6, 10, [np.arange(k) for k in (1, 3, 0, 2, 4, 2)], rng)
    bad_col.col_idx = bad_col.col_idx.copy()
    bad_col.col_idx[4] = 10  # one column index == n
    bad_rp = _csr(pkg, 6, 10, [np.arange(k) for k in (1, 3, 0, 2, 4, 2)], rng)
    bad_rp.row_ptr = bad_rp.row_ptr.copy()
    bad_rp.row_ptr[3] = bad_rp.row_ptr[2] - 1  # a decreasing row pointer
    for p in (bad_col, bad_rp):
        with pytest.raises(pkg.PdhgError):
            pkg.csr_spmv(p, 1.0, x_t, 0.0, np.zeros(10), transpose=True)
        assert np.isnan(_call(pkg, p, True, 1.0, x_t, 0.0, y_t)).all()
        assert np.isnan(_call(pkg, p, False, 1.0, y_t, 0.0, x_t)).all()
    # a row pointer whose end disagrees with nnz
    assert np.isnan(_call(pkg, good, True, 1.0, x_t, 0.0, y_t, nnz=good.nnz - 1)).all()
    # the next well-formed call clears the flag
    got = _call(pkg, good, True, 1.0, x_t, 0.0, y_t)
    assert np.array_equal(got, pkg.csr_spmv(good, 1.0, x_t, 0.0, np.zeros(10), transpose=True))


def test_noalloc_spmv_refuses_sizes_beyond_its_scratch(pkg):
    f = _entry(pkg)
    rp = np.zeros(2, dtype=np.int32)
    # 300,000 columns exceed the 262,144 the fixed scratch holds; refused before any work
    rc = f(1, 1, 300_000, 0, rp.ctypes.data, None, None, 1.0, None, 0.0, rp.ctypes.data, None)
    assert rc == PDHG_ERR_INVALID_ARGUMENT
    rc = f(1, 10, 100, 300_000, rp.ctypes.data, rp.ctypes.data, rp.ctypes.data, 1.0,
           rp.ctypes.data, 0.0, rp.ctypes.data, None)
    assert rc == PDHG_ERR_INVALID_ARGUMENT
