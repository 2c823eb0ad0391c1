"""The iteration-kernel autotuner: it times the candidate shapes on a large
LP, keeps valid ones, leaves results unchanged within the mixed-mode
tolerance, and persists its choices in the JSON cache file when asked."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KW = dict(precision="mixed", termination_rule="relative_kkt", restart_rule="adaptive",
          max_iterations=200_000)


def test_autotune_picks_valid_shapes_and_keeps_the_optimum(pkg):
    p = pkg.lpgen.transportation_lp(500, 1100, seed=1000)  # 1.1M nonzeros
    assert p.nnz >= 1 << 20
    with pkg.Engine(0) as e:
        e.load(p)
        assert not e.tuning("mixed")["timed"]
        tuned = e.solve(pkg.PdhgOptions(**KW))
        t = e.tuning("mixed")
        assert t["timed"]
        for k in ("primal_lanes", "dual_lanes"):
            assert t[k] in (1, 2, 4, 8, 16, 32)
        assert t["primal_long_mode"] in (0, 1, 2) and t["dual_long_mode"] in (0, 1, 2)
        fixed = e.solve(pkg.PdhgOptions(autotune=False, **KW))
    assert tuned.status == fixed.status == "optimal"
    assert abs(tuned.objective - fixed.objective) <= 2e-3 * abs(fixed.objective)


SNIPPET = """
import importlib, json, sys
sys.path.insert(0, {root!r})
pkg = importlib.import_module("sovereign-solver_b200")
p = pkg.lpgen.transportation_lp(500, 1100, seed=1000)
with pkg.Engine(0) as e:
    e.load(p)
    e.solve(pkg.PdhgOptions(precision="mixed", max_iterations=40))
    print(json.dumps(e.tuning("mixed")))
"""


def test_tuning_cache_file_is_written_and_reused(tmp_path):
    cache = tmp_path / "tune.json"
    env = dict(os.environ, PDHG_B200_TUNE_CACHE=str(cache))
    code = SNIPPET.format(root=ROOT)
    first = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                           text=True, timeout=600)
    assert first.returncode == 0, first.stderr
    entries = json.loads(cache.read_text())
    assert any(k.startswith("f32/primal/") for k in entries)
    assert any(k.startswith("f32/dual/") for k in entries)
    # a fresh process takes the shapes from the file
    second = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                            text=True, timeout=600)
    assert second.returncode == 0, second.stderr
    assert json.loads(first.stdout.strip().splitlines()[-1]) == \
        json.loads(second.stdout.strip().splitlines()[-1])
