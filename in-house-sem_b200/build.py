"""Builds the CUDA backend library ``lib/libinsem_cuda.so`` in-tree for sm_100a.

Each translation unit is compiled by its own nvcc process (the element
kernels once per number of GLL points), in parallel, then linked into one
shared library that exports the C ABI of ``include/insem_cuda.h``.

    python in-house-sem_b200/build.py [--jobs N] [--verbose]
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build" / "obj"
LIB = PKG / "lib" / "libinsem_cuda.so"
CASES_LIB = PKG / "lib" / "libinsem_cases.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr", "--default-stream", "per-thread",
    "-Xcompiler", "-fPIC,-O3", "-I", str(REPO / "include"),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def units() -> list[tuple[Path, list[str], Path]]:
    """(source, extra flags, object) for every translation unit."""
    out = []
    for ng in range(2, 10):
        out.append((CSRC / "element_ng.cu", [f"-DINSEM_NG={ng}"], OBJ / f"element_ng{ng}.o"))
        out.append((CSRC / "tiled_ng.cu", [f"-DINSEM_NG={ng}"], OBJ / f"tiled_ng{ng}.o"))
    for name in ("seams.cu", "solver.cu", "tiled_path.cu", "batch.cu", "snapshots.cu", "noalloc.cu"):
        if (CSRC / name).exists():
            out.append((CSRC / name, [], OBJ / (Path(name).stem + ".o")))
    return out


def newest_header() -> float:
    return max(p.stat().st_mtime for p in list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp"))
               + [REPO / "include" / "insem_cuda.h"])


def compile_unit(src: Path, extra: list[str], obj: Path, verbose: bool, force: bool) -> str:
    if not force and obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, newest_header()):
        return f"up to date {obj.name}"
    obj.parent.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name} {' '.join(extra)}:\n{res.stderr[-6000:]}")
    return res.stderr if verbose else f"built {obj.name}"


def build_cases(force: bool = False) -> Path:
    """Host-only case-setup library (csrc/host), compiled with the system C++
    compiler.  No contraction to fused multiply-adds, so every double the
    setup forms rounds like the reference's setup code."""
    host = CSRC / "host"
    srcs = sorted(host.glob("*.cpp"))
    newest = max(p.stat().st_mtime for p in srcs + sorted(host.glob("*.h")) + sorted(host.glob("*.hpp")))
    if force or not CASES_LIB.exists() or CASES_LIB.stat().st_mtime < newest:
        CASES_LIB.parent.mkdir(parents=True, exist_ok=True)
        cxx = shutil.which("g++") or "c++"
        tmp = CASES_LIB.with_suffix(".so.tmp")
        cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-ffp-contract=off",
               *[str(s) for s in srcs], "-o", str(tmp)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"case library build failed:\n{res.stderr[-6000:]}")
        tmp.replace(CASES_LIB)
    return CASES_LIB


def build(jobs: int | None = None, verbose: bool = False, force: bool = False) -> Path:
    jobs = jobs or max(1, min(16, os.cpu_count() or 1))
    build_cases(force)
    todo = units()
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        logs = list(ex.map(lambda u: compile_unit(*u, verbose, force), todo))
    if verbose:
        for line in logs:
            print(line)
    objs = [str(o) for _, _, o in todo]
    if force or not LIB.exists() or LIB.stat().st_mtime < max(Path(o).stat().st_mtime for o in objs):
        LIB.parent.mkdir(parents=True, exist_ok=True)
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
        tmp.replace(LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(args.jobs, args.verbose, args.force))


if __name__ == "__main__":
    sys.exit(main())
