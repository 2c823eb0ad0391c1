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
