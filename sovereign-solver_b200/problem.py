"""The LP the engine consumes, in the reference's canonical form.

Mirrors ``sov::Problem`` (include/sovereign/problem.hpp:47-127):

    optimize   c^T x + obj_const          (minimize, or maximize)
    subject to row_lo <= A x <= row_hi,   col_lo <= x <= col_hi

``A`` is CSR with int32 indices (``Idx`` is int32 unless the reference is built
with SOVEREIGN_INDEX64, include/sovereign/numeric.hpp:65-71), strictly
ascending column indices inside each row, FP64 values. Infinite bounds are
``+-inf`` (``kInfinity``, problem.hpp:29).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

INF = float("inf")


@dataclass
class Problem:
    m: int
    n: int
    row_ptr: np.ndarray  # int32, m+1
    col_idx: np.ndarray  # int32, nnz
    val: np.ndarray  # float64, nnz
    c: np.ndarray  # float64, n
    col_lo: np.ndarray  # float64, n
    col_hi: np.ndarray  # float64, n
    row_lo: np.ndarray  # float64, m
    row_hi: np.ndarray  # float64, m
    obj_const: float = 0.0
    maximize: bool = False
    name: str = ""

    def __post_init__(self) -> None:
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int32)
        self.col_idx = np.ascontiguousarray(self.col_idx, dtype=np.int32)
        for f in ("val", "c", "col_lo", "col_hi", "row_lo", "row_hi"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float64))
        self.m = int(self.m)
        self.n = int(self.n)

    @property
    def nnz(self) -> int:
        return int(self.col_idx.shape[0])

    def evaluate_objective(self, x: np.ndarray) -> float:
        """``Problem::evaluate_objective`` (src/io/problem.cpp:13-19): sequential sum."""
        acc = float(self.obj_const)
        for cj, xj in zip(self.c.tolist(), np.asarray(x, dtype=np.float64).tolist()):
            acc += cj * xj
        return acc

    def to_dict(self) -> dict:
        return {
            "m": self.m, "n": self.n, "row_ptr": self.row_ptr, "col_idx": self.col_idx,
            "val": self.val, "c": self.c, "col_lo": self.col_lo, "col_hi": self.col_hi,
            "row_lo": self.row_lo, "row_hi": self.row_hi, "obj_const": self.obj_const,
            "maximize": self.maximize,
        }

    @staticmethod
    def from_dict(d) -> "Problem":
        return Problem(
            m=int(d["m"]), n=int(d["n"]), row_ptr=d["row_ptr"], col_idx=d["col_idx"],
            val=d["val"], c=d["c"], col_lo=d["col_lo"], col_hi=d["col_hi"],
            row_lo=d["row_lo"], row_hi=d["row_hi"], obj_const=float(d["obj_const"]),
            maximize=bool(d["maximize"]))

    @staticmethod
    def from_coo(m: int, n: int, rows, cols, vals, **kw) -> "Problem":
        """CSR from (row, col, value) triplets with distinct (row, col) pairs."""
        rows = np.asarray(rows, dtype=np.int64)
        cols = np.asarray(cols, dtype=np.int64)
        vals = np.asarray(vals, dtype=np.float64)
        order = np.lexsort((cols, rows))
        rows, cols, vals = rows[order], cols[order], vals[order]
        if rows.size > 1:
            dup = (rows[1:] == rows[:-1]) & (cols[1:] == cols[:-1])
            if dup.any():
                raise ValueError("from_coo: repeated (row, col) entry")
        counts = np.bincount(rows, minlength=m) if rows.size else np.zeros(m, np.int64)
        row_ptr = np.zeros(m + 1, dtype=np.int64)
        np.cumsum(counts, out=row_ptr[1:])
        return Problem(m=m, n=n, row_ptr=row_ptr, col_idx=cols, val=vals, **kw)
