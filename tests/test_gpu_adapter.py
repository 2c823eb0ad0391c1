"""Drop-in check: the reference's own types driving the B200 engine.

oracle/_ref/adapter_check (built by oracle/Makefile from tests/cpp/
adapter_check.cpp against the reference's headers and compiled PDHG path)
solves LPs built with sov::Problem::Builder through the reference's sov::Pdhg
on its Host backend and through sov::PdhgB200 (include/pdhg_b200_sov.hpp, the
engine behind the same interface), and requires identical results, messages,
checkpoint calls and cancellation behaviour.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "adapter_check")


def test_reference_interface_over_the_engine_is_bit_identical():
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/adapter_check not built (needs the reference sources)")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ALL OK" in r.stdout, r.stdout + r.stderr
