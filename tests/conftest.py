"""Shared test setup: paths, the `gpu` marker, golden-fixture loading."""
from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built engine library")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("sovereign-solver_b200")


@pytest.fixture(scope="session")
def orc():
    import orc as _orc
    return _orc


def golden_names(prefix: str = "") -> list[str]:
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and f.startswith(prefix))


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False) as z:
        out = {}
        for k in z.files:
            v = z[k]
            out[k] = v.item() if v.ndim == 0 else v
    if "options_json" in out:
        out["options"] = json.loads(out.pop("options_json"))
    return out


def golden_problem(pkg, g: dict):
    return pkg.Problem.from_dict(g)


PDHG_CASES = [n for n in golden_names() if n.startswith(("pdhg_", "smoke_", "rand_", "mixed_", "c0_"))]


def highs_optimum(p):
    """The LP's optimal objective from scipy's HiGHS (an independent exact
    solver, for checking the objectives of solutions at a relative-KKT
    tolerance)."""
    from scipy.optimize import linprog
    A = np.zeros((p.m, p.n))
    for i in range(p.m):
        for k in range(p.row_ptr[i], p.row_ptr[i + 1]):
            A[i, p.col_idx[k]] += p.val[k]
    eq = np.isfinite(p.row_lo) & np.isfinite(p.row_hi) & (p.row_lo == p.row_hi)
    ub_rows, ub_rhs = [], []
    for i in np.nonzero(~eq)[0]:
        if np.isfinite(p.row_hi[i]):
            ub_rows.append(A[i]); ub_rhs.append(p.row_hi[i])
        if np.isfinite(p.row_lo[i]):
            ub_rows.append(-A[i]); ub_rhs.append(-p.row_lo[i])
    sgn = -1.0 if p.maximize else 1.0
    res = linprog(sgn * p.c, A_ub=np.array(ub_rows) if ub_rows else None,
                  b_ub=np.array(ub_rhs) if ub_rhs else None,
                  A_eq=A[eq] if eq.any() else None, b_eq=p.row_lo[eq] if eq.any() else None,
                  bounds=list(zip(np.where(np.isfinite(p.col_lo), p.col_lo, None),
                                  np.where(np.isfinite(p.col_hi), p.col_hi, None))),
                  method="highs")
    assert res.status == 0, res.message
    return sgn * res.fun + p.obj_const
