"""Times the reference's own CPU time loop (oracle build, libbench_ref.so).

TEST / BENCHMARK INFRASTRUCTURE ONLY: bench.py's reference arm and CPU
baseline leg.  The model is passed as the same description the backend's
native setup takes (insem_b200.cases.describe); the reference builds it
through its own C++ API (oracle/ref/bench_ref.cpp) and runs
Solver::advance with OpenMP on the host cores.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "float" / "libbench_ref.so"


def available() -> bool:
    return LIB.exists()


def run(model, dt: float, warmup: int, steps: int) -> dict:
    """Builds `model` with the reference and times `steps` steps after `warmup`."""
    from insem_b200 import cases as K

    L = C.CDLL(str(LIB))
    L.bench_ref_run.argtypes = [C.c_void_p, C.c_double, C.c_int32, C.c_int32, C.POINTER(C.c_double)]
    L.bench_ref_run.restype = C.c_int
    L.bench_ref_last_error.restype = C.c_char_p
    desc, keep = K.describe(model)
    out = (C.c_double * 5)()
    if L.bench_ref_run(C.byref(desc), dt, warmup, steps, out) != 0:
        raise RuntimeError("reference run failed: " + L.bench_ref_last_error().decode())
    return {"seconds": out[0], "setup_seconds": out[1], "points": out[2], "dt": out[3], "elements": int(out[4])}
