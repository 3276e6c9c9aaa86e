"""The reference arm of bench.py (LatticeQM's :multithreaded density-matrix k-loop
restated in C++/OpenMP, oracle/cpu_kspace.cpp) prints one JSON line with the keys
the throughput line carries; under several ranks only rank 0 prints.  Host-only:
one warm-up and one timed step, one k-point per host thread (about 10 s)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_arm(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return [ln for ln in p.stdout.splitlines() if ln.startswith("{")]


@pytest.fixture(scope="module")
def line():
    sys.path.insert(0, ROOT)
    from oracle import build_cpu
    build_cpu.build()
    lines = run_arm({"RANK": "0", "WORLD_SIZE": "1"})
    assert len(lines) == 1
    return json.loads(lines[0])


def test_reference_arm_line_keys(line):
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "k-pts/s" and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["dtype"] == "f64"
    assert "workload" in line["config"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_prints_nothing_on_other_ranks():
    assert run_arm({"RANK": "1", "WORLD_SIZE": "2"}) == []
