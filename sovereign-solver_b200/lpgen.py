"""Seeded synthetic LP families (the workloads the engine is measured on).

No public instance suite is available offline, so every workload is a seeded
random LP of a fixed shape. Seeds are ``1000 * family + instance``. Each
generator returns a :class:`Problem` with strictly ascending, duplicate-free
CSR rows (column nonzero rows are drawn WITHOUT replacement, so nothing is
summed when the reference's ``CsrMatrix::from_triplets`` rebuilds the matrix,
src/l0/sparse.cpp:30-70).

Families:
  random_equality_lp      m equality rows, n columns, k N(0,1) nonzeros per
                          column at uniform rows; 0 <= x <= 10; b = A x0 with
                          x0 ~ U[0,10]; c = A^T y0 + s, y0 ~ N(0,1), s ~ U[0,1].
                          (2,000 x 5,000, k=5: the small single-LP case.)
  transportation_lp       S supplies x D demands; supply rows sum_j x_ij <= S_i,
                          demand rows sum_i x_ij >= D_j, every value 1.0;
                          S ~ U[50,150] rescaled to 1.05 x total demand,
                          D ~ U[20,60], cost ~ U[1,100], x >= 0.
                          (2,000 x 5,000 = 10M columns, 7,000 rows, 20M nonzeros.)
  badly_scaled_lp         Zipf(s=1.1) row popularity, |a| log-uniform in
                          [1e-3, 1e3] with random signs, 30% <= rows;
                          -U[0,5] <= x <= U[0,5].
  batch_family            instances of random_equality_lp structure with
                          m = floor(exp(U[ln 50, ln 5000])), n = m * U{2,3},
                          U{4..10} nonzeros per column.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .problem import INF, Problem


def _distinct_rows(rng: np.random.Generator, n: int, k: int, m: int,
                   p: np.ndarray | None = None) -> np.ndarray:
    """An (n, k) array of row indices, distinct within each column."""
    if k > m:
        raise ValueError("more nonzeros per column than rows")
    if p is None:
        rows = rng.integers(0, m, size=(n, k))
    else:
        rows = rng.choice(m, size=(n, k), p=p)
    for _ in range(10_000):
        s = np.sort(rows, axis=1)
        dup_sorted = np.zeros_like(s, dtype=bool)
        dup_sorted[:, 1:] = s[:, 1:] == s[:, :-1]
        bad_cols = np.nonzero(dup_sorted.any(axis=1))[0]
        if bad_cols.size == 0:
            return rows
        # Redraw the later duplicates of each bad column.
        sub = rows[bad_cols]
        order = np.argsort(sub, axis=1, kind="stable")
        ss = np.take_along_axis(sub, order, axis=1)
        d = np.zeros_like(ss, dtype=bool)
        d[:, 1:] = ss[:, 1:] == ss[:, :-1]
        redraw = np.zeros_like(d)
        np.put_along_axis(redraw, order, d, axis=1)
        cnt = int(redraw.sum())
        if p is None:
            sub[redraw] = rng.integers(0, m, size=cnt)
        else:
            sub[redraw] = rng.choice(m, size=cnt, p=p)
        rows[bad_cols] = sub
    raise RuntimeError("could not draw distinct rows")


def _csr_from_columns(m: int, n: int, rows: np.ndarray, vals: np.ndarray, **kw) -> Problem:
    """CSR from per-column (row, value) lists; rows (n, k) distinct per column."""
    k = rows.shape[1]
    cols = np.repeat(np.arange(n, dtype=np.int64), k)
    r = rows.reshape(-1).astype(np.int64)
    v = vals.reshape(-1)
    order = np.lexsort((cols, r))
    r, cols, v = r[order], cols[order], v[order]
    counts = np.bincount(r, minlength=m)
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return Problem(m=m, n=n, row_ptr=row_ptr, col_idx=cols, val=v, **kw)


def random_equality_lp(m: int = 2000, n: int = 5000, k: int = 5, seed: int = 0,
                       maximize: bool = False) -> Problem:
    rng = np.random.default_rng(seed)
    rows = _distinct_rows(rng, n, k, m)
    vals = rng.standard_normal((n, k))
    A = _csr_from_columns(m, n, rows, vals, c=np.zeros(n), col_lo=np.zeros(n),
                          col_hi=np.full(n, 10.0), row_lo=np.zeros(m), row_hi=np.zeros(m),
                          maximize=maximize, name=f"random_equality_{m}x{n}_s{seed}")
    x0 = rng.uniform(0.0, 10.0, n)
    y0 = rng.standard_normal(m)
    s = rng.uniform(0.0, 1.0, n)
    b = csr_matvec(A, x0)
    c = csr_rmatvec(A, y0) + s
    A.row_lo = b.copy()
    A.row_hi = b.copy()
    A.c = -c if maximize else c
    return A


def transportation_lp(supplies: int = 2000, demands: int = 5000, seed: int = 1000) -> Problem:
    rng = np.random.default_rng(seed)
    S, D = supplies, demands
    dem = rng.uniform(20.0, 60.0, D)
    sup = rng.uniform(50.0, 150.0, S)
    sup *= 1.05 * dem.sum() / sup.sum()
    cost = rng.uniform(1.0, 100.0, S * D)
    m, n = S + D, S * D
    nnz = 2 * n
    row_ptr = np.empty(m + 1, dtype=np.int64)
    row_ptr[: S + 1] = np.arange(S + 1, dtype=np.int64) * D
    row_ptr[S + 1:] = S * D + np.arange(1, D + 1, dtype=np.int64) * S
    col_idx = np.empty(nnz, dtype=np.int32)
    col_idx[: S * D] = np.arange(S * D, dtype=np.int32)  # supply row i: i*D .. i*D+D-1
    # demand row j: j, D+j, 2D+j, ...
    col_idx[S * D:] = (np.arange(S, dtype=np.int64)[None, :] * D
                       + np.arange(D, dtype=np.int64)[:, None]).reshape(-1).astype(np.int32)
    row_lo = np.concatenate([np.full(S, -INF), dem])
    row_hi = np.concatenate([sup, np.full(D, INF)])
    return Problem(m=m, n=n, row_ptr=row_ptr, col_idx=col_idx, val=np.ones(nnz), c=cost,
                   col_lo=np.zeros(n), col_hi=np.full(n, INF), row_lo=row_lo, row_hi=row_hi,
                   name=f"transportation_{S}x{D}_s{seed}")


def badly_scaled_lp(m: int = 200_000, n: int = 500_000, k: int = 8, seed: int = 2000,
                    zipf_s: float = 1.1, ineq_frac: float = 0.3) -> Problem:
    return _badly_scaled_with_point(m, n, k, seed, zipf_s, ineq_frac)[0]


def _badly_scaled_with_point(m: int, n: int, k: int, seed: int, zipf_s: float = 1.1,
                             ineq_frac: float = 0.3):
    """badly_scaled_lp and the interior point x0 its b was built from."""
    rng = np.random.default_rng(seed)
    ranks = rng.permutation(m) + 1
    p = ranks.astype(np.float64) ** (-zipf_s)
    p /= p.sum()
    rows = _distinct_rows(rng, n, k, m, p=p)
    mag = np.exp(rng.uniform(math.log(1e-3), math.log(1e3), (n, k)))
    sign = np.where(rng.random((n, k)) < 0.5, -1.0, 1.0)
    A = _csr_from_columns(m, n, rows, mag * sign, c=np.zeros(n), col_lo=np.zeros(n),
                          col_hi=np.zeros(n), row_lo=np.zeros(m), row_hi=np.zeros(m),
                          name=f"badly_scaled_{m}x{n}_s{seed}")
    lo = -rng.uniform(0.0, 5.0, n)
    hi = rng.uniform(0.0, 5.0, n)
    x0 = lo + (hi - lo) * rng.uniform(0.0, 1.0, n)
    ineq = rng.random(m) < ineq_frac
    ax = csr_matvec(A, x0)
    b = ax + np.where(ineq, rng.uniform(0.0, 1.0, m), 0.0)
    y0 = rng.standard_normal(m)
    y0 = np.where(ineq, -np.abs(y0), y0)
    s = rng.uniform(0.0, 1.0, n)
    A.c = csr_rmatvec(A, y0) + s
    A.col_lo, A.col_hi = lo, hi
    A.row_lo = np.where(ineq, -INF, b)
    A.row_hi = b
    return A, x0


def row_lengths_lp(lengths: list[int], n: int, seed: int = 0) -> Problem:
    """Equality LP of config-0 structure whose row i has exactly lengths[i]
    nonzeros (distinct random columns), to exercise every row-length tier of
    the kernels (short rows, warp rows, CTA rows)."""
    rng = np.random.default_rng(seed)
    m = len(lengths)
    cols = [np.sort(rng.choice(n, size=k, replace=False)) for k in lengths]
    row_ptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum([len(c) for c in cols], out=row_ptr[1:])
    col_idx = np.concatenate(cols).astype(np.int64)
    val = rng.standard_normal(col_idx.size)
    A = Problem(m=m, n=n, row_ptr=row_ptr, col_idx=col_idx, val=val, c=np.zeros(n),
                col_lo=np.zeros(n), col_hi=np.full(n, 10.0), row_lo=np.zeros(m),
                row_hi=np.zeros(m), name=f"row_lengths_{m}x{n}_s{seed}")
    x0 = rng.uniform(0.0, 10.0, n)
    y0 = rng.standard_normal(m)
    b = csr_matvec(A, x0)
    A.row_lo = b.copy()
    A.row_hi = b.copy()
    A.c = csr_rmatvec(A, y0) + rng.uniform(0.0, 1.0, n)
    return A


@dataclasses.dataclass
class ParametricFamily:
    """A parametric LP family over one matrix: b = b0 + B_b theta and
    c = c0 + B_c theta (theta in R^p), the <= rows of the base staying <=."""
    base: Problem
    Bb: np.ndarray      # m x p
    Bc: np.ndarray      # n x p
    ineq: np.ndarray    # rows with row_lo = -inf
    theta_std: float

    @property
    def n_params(self) -> int:
        return self.Bb.shape[1]

    def instance(self, theta: np.ndarray) -> Problem:
        b = self.base.row_hi + self.Bb @ theta
        c = self.base.c + self.Bc @ theta
        return dataclasses.replace(self.base, c=c, row_lo=np.where(self.ineq, -INF, b),
                                   row_hi=b, name=f"{self.base.name}_theta")

    def thetas(self, count: int, seed: int) -> np.ndarray:
        rng = np.random.default_rng(seed)
        return rng.normal(0.0, self.theta_std, (count, self.n_params))


def parametric_family(m: int = 50_000, n: int = 120_000, k: int = 5, seed: int = 4000,
                      n_params: int = 64, rel: float = 0.1, theta_std: float = 0.1,
                      b_mode: str = "feasible", box_frac: float = 0.1) -> ParametricFamily:
    """Config 4: the base is config-2 structure (power-law rows, log-uniform
    magnitudes, 30% <= rows, box bounds, b = A x0 (+ slack) for an interior
    x0); theta ~ N(0, theta_std^2 I). B_c is dense Gaussian with
    E||B_c theta|| = rel ||c0|| (every c is bounded over the box).

    b_mode "gaussian": B_b dense Gaussian with E||B_b theta|| = rel ||b0||. On
    badly scaled bases with equality rows and boxes this makes (nearly) every
    instance infeasible. b_mode "feasible" (default): B_b = A B_x, i.e. b moves
    with a feasible point x0 + B_x theta, B_x dense Gaussian with each row
    scaled so the point's coordinate moves with a standard deviation of
    box_frac times its distance to the nearer bound."""
    base, x0 = _badly_scaled_with_point(m, n, k, seed)
    rng = np.random.default_rng(seed + 1)
    Bc = rng.standard_normal((n, n_params))
    Bc *= rel * np.linalg.norm(base.c) / (theta_std * np.linalg.norm(Bc))
    if b_mode == "gaussian":
        Bb = rng.standard_normal((m, n_params))
        Bb *= rel * np.linalg.norm(base.row_hi) / (theta_std * np.linalg.norm(Bb))
    elif b_mode == "feasible":
        Bx = rng.standard_normal((n, n_params))
        dist = np.minimum(x0 - base.col_lo, base.col_hi - x0)
        Bx *= (box_frac * dist / (theta_std * np.linalg.norm(Bx, axis=1)))[:, None]
        Bb = np.stack([csr_matvec(base, Bx[:, j]) for j in range(n_params)], axis=1)
    else:
        raise ValueError(b_mode)
    ineq = ~np.isfinite(base.row_lo)
    return ParametricFamily(base=base, Bb=Bb, Bc=Bc, ineq=ineq, theta_std=theta_std)


def batch_family(count: int = 4096, seed_base: int = 3000, m_lo: int = 50,
                 m_hi: int = 5000) -> list[Problem]:
    out = []
    for inst in range(count):
        rng = np.random.default_rng(seed_base + inst)
        m = int(math.floor(math.exp(rng.uniform(math.log(m_lo), math.log(m_hi)))))
        n = m * int(rng.integers(2, 4))
        k = int(rng.integers(4, 11))
        out.append(random_equality_lp(m, n, min(k, m), seed=int(rng.integers(1 << 31))))
    return out


def csr_matvec(p: Problem, x: np.ndarray) -> np.ndarray:
    prod = p.val * x[p.col_idx]
    out = np.zeros(p.m)
    lengths = np.diff(p.row_ptr)
    nz = lengths > 0
    out[nz] = np.add.reduceat(prod, p.row_ptr[:-1][nz]) if prod.size else 0.0
    return out


def csr_rmatvec(p: Problem, y: np.ndarray) -> np.ndarray:
    rows = np.repeat(np.arange(p.m), np.diff(p.row_ptr))
    return np.bincount(p.col_idx, weights=p.val * y[rows], minlength=p.n)
