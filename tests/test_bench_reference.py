"""The bench's reference arm (the reference's own CPU integrator, oracle/_ref) on CPU: the JSON
line it prints carries the contract's keys, and ranks other than 0 exit without work."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "detector_1024",
                           "--steps", "2", "--warmup", "1"], cwd=REPO, env=env, capture_output=True, text=True,
                          timeout=600)


def test_reference_arm_prints_one_contract_line():
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref is not built (the reference's C sources are absent)")
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "caked_frames_per_s" and d["unit"] == "frames/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("detector_1024")


def test_reference_arm_other_ranks_exit_without_output():
    r = _run({"RANK": "1"})
    assert r.returncode == 0
    assert not any(ln.startswith("{") for ln in r.stdout.splitlines())
