"""The tile kernels' shared-memory layout, checked on the host: the element
data region is reused for the xi-flux rows and then for the assembly target
with v and 1/M, so regions that are live together must never overlap, and
every bulk-copy destination must be 16-byte aligned.  Compiles
tests/layout_check.cu (host code only) with the library's own flags and runs
it over every ngll, geometry kind, medium, order and tile size."""

from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def test_shared_memory_layout_invariants(tmp_path):
    sys.path.insert(0, str(REPO / "in-house-sem_b200"))
    try:
        import build
    finally:
        sys.path.pop(0)
    try:
        nvcc = build.nvcc()
    except RuntimeError:
        pytest.skip("nvcc not available")
    if not shutil.which(nvcc) and not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    exe = tmp_path / "layout_check"
    cmd = [nvcc, *build.NVCC_FLAGS, "-I", str(build.CSRC), str(REPO / "tests" / "layout_check.cu"), "-o", str(exe)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.startswith("ok"), run.stdout + run.stderr
