"""The benchmark's reference arm on the CPU: the oracle port on every host core (spawned worker
processes, each with its own factorisations), on a small torus, printing the bench contract's line."""

from __future__ import annotations

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_uses_the_host_cores_and_prints_its_line() -> None:
    result = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
         "--cols", "32", "--rows", "16", "--queries", "8"],
        capture_output=True, text=True, timeout=600, cwd=ROOT,
    )
    assert result.returncode == 0, result.stderr[-2000:]
    line = json.loads([l for l in result.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "solves/s"
    cores = line["cpu_baseline"]["cores"]
    assert 1 <= cores <= min(len(os.sched_getaffinity(0)), 8)
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
