"""bench.py's reference arm: it runs the reference's own CPU time loop (the
oracle/_ref build of the reference sources) and prints one JSON line in the
contract's shape, timing exactly --steps steps after --warmup."""

from __future__ import annotations

import json
import subprocess
import sys

import pytest

from conftest import REPO


def test_reference_arm_line(pkg):
    sys.path.insert(0, str(REPO))
    try:
        from oracle import refbench
    finally:
        sys.path.pop(0)
    if not refbench.available():
        pytest.skip("reference build (oracle/_ref) not present")
    res = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "2", "--warmup", "3"],
                         capture_output=True, text=True, timeout=600, cwd=str(REPO))
    assert res.returncode == 0, res.stderr[-3000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert line["metric"] == "GLL-point-updates/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
