"""The seeded workload generators: shapes, CSR validity, determinism."""
import numpy as np
import pytest


def _valid_csr(p):
    assert p.row_ptr[0] == 0 and p.row_ptr[-1] == p.nnz
    assert np.all(np.diff(p.row_ptr) >= 0)
    for r in range(min(p.m, 200)):
        cols = p.col_idx[p.row_ptr[r]:p.row_ptr[r + 1]]
        assert np.all(np.diff(cols) > 0)
    assert p.col_idx.min() >= 0 and p.col_idx.max() < p.n
    assert np.isfinite(p.val).all()


def test_random_equality_shape_and_feasibility(pkg):
    p = pkg.lpgen.random_equality_lp(200, 500, 5, seed=0)
    _valid_csr(p)
    assert p.nnz == 2500  # 5 distinct rows per column
    assert np.array_equal(p.row_lo, p.row_hi)
    assert (p.col_lo == 0).all() and (p.col_hi == 10).all()
    q = pkg.lpgen.random_equality_lp(200, 500, 5, seed=0)
    assert np.array_equal(p.val, q.val) and np.array_equal(p.c, q.c)


def test_transportation_structure(pkg):
    p = pkg.lpgen.transportation_lp(20, 50, seed=1000)
    _valid_csr(p)
    assert (p.m, p.n, p.nnz) == (70, 1000, 2000)
    assert (p.val == 1.0).all()
    counts = np.bincount(p.col_idx, minlength=p.n)
    assert (counts == 2).all()
    supply, demand = p.row_hi[:20], p.row_lo[20:]
    assert abs(supply.sum() - 1.05 * demand.sum()) < 1e-6 * supply.sum()
    assert np.isinf(p.row_lo[:20]).all() and np.isinf(p.row_hi[20:]).all()


def test_badly_scaled_structure(pkg):
    p = pkg.lpgen.badly_scaled_lp(2000, 5000, 8, seed=2000)
    _valid_csr(p)
    mag = np.abs(p.val)
    assert mag.min() >= 1e-3 * (1 - 1e-12) and mag.max() <= 1e3 * (1 + 1e-12)
    lengths = np.diff(p.row_ptr)
    assert lengths.max() > 20 * np.median(lengths)  # power-law rows
    ineq = np.isinf(p.row_lo)
    assert 0.2 < ineq.mean() < 0.4
    assert (p.col_lo <= 0).all() and (p.col_hi >= 0).all()


def test_batch_family_ranges(pkg):
    probs = pkg.lpgen.batch_family(12, seed_base=3000)
    for p in probs:
        _valid_csr(p)
        assert 50 <= p.m <= 5000 and p.n in (2 * p.m, 3 * p.m)
