"""The native case builder against the reference's setup on the benchmarked models (CPU only).

``tests/golden/timed_<case>.npz`` holds a SHA-256 digest of every array the
reference solver packed for the models of ``tests/golden/timed_models.py``:
config 2 at its stated geometry, config 3 at 64 x 64 elements, six of the 256
config 4 boreholes that ``bench.py`` times, and the Gaussian / sampled source
time function cases.  Every array the native builder produces must hash to the
same digest once cast to the reference's dtype (integers exactly, floats bit
for bit).
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import GOLDEN

TIMED = ["c2", "c3s", "stfg", "stfs", "snapbh1", "snaplay", "c4m0", "c4m1", "c4m12", "c4m17", "c4m72", "c4m80"]
SKIP = ("problem.dt", "problem.stable_dt", "problem.n_steps", "problem.real_bytes")


def timed_fixture(case):
    return np.load(GOLDEN / f"timed_{case}.npz")


def timed_model(case):
    import sys

    sys.path.insert(0, str(GOLDEN))
    import timed_models

    return timed_models.TIMED[case]()


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", TIMED)
def test_builder_matches_reference_on_benchmarked_models(pkg, case):
    from insem_b200 import cases as K

    z = timed_fixture(case)
    model, _, _ = timed_model(case)
    arrays = K.setup_arrays(model)
    checked, mismatched = 0, []
    for hk in z.files:
        if not hk.startswith("hash.problem."):
            continue
        key = hk[len("hash."):]
        if key in SKIP or key.endswith(".coords") or key.endswith("trace_index"):
            continue
        size = int(z[f"size.{key}"])
        if key not in arrays:
            assert size == 0, f"{key}: the builder has no array, the reference has {size} entries"
            continue
        v = np.asarray(arrays[key])
        assert v.size == size, (key, v.size, size)
        v = v.astype(np.dtype(str(z[f"dtype.{key}"])))
        if digest(v) != str(z[hk]):
            mismatched.append(key)
        checked += 1
    assert not mismatched, f"arrays differing from the reference's setup: {mismatched[:8]}"
    assert checked > 20


# Error of the float build (and so of the CUDA path, which equals it bit for
# bit) against the FP64 build (INSEM_REAL=double) on the benchmarked models,
# as stated in the design notes: worst receiver-trace relative L2 error, and
# the float build's total energy against the FP64 build's, relative to the
# largest FP64 energy.  Both builds run the same dt and steps.
FP64_BOUNDS = {  # case: (trace rel-L2, energy)
    "c2": (2e-5, 3e-6), "c3s": (6e-5, 3e-6), "c4m0": (2e-5, 6e-6), "c4m1": (8e-5, 1e-6),
    "c4m12": (2e-5, 1e-6), "c4m17": (3e-5, 1e-6), "c4m72": (6e-5, 3e-6), "c4m80": (3e-5, 1e-6),
    "stfg": (4e-4, 1e-6), "stfs": (1e-6, 1e-6), "snapbh1": (3e-6, None), "snaplay": (3e-6, None),
}


@pytest.mark.parametrize("case", TIMED)
def test_float_build_error_against_fp64(case):
    import golden_io as G

    z, d = timed_fixture(case), np.load(GOLDEN / f"timed_{case}_f64.npz")
    assert float(z["meta.dt"]) == float(d["meta.dt"]) and int(z["meta.n_steps_run"]) == int(d["meta.n_steps_run"])
    worst = max(G.rel_l2(z[k], d[k]) for k in z.files if k.startswith("run.trace."))
    trace_bound, energy_bound = FP64_BOUNDS[case]
    assert worst <= trace_bound, worst
    if energy_bound is not None:  # the model records the energy monitor
        e32, e64 = z["run.energy"], d["run.energy"]
        tot32, tot64 = e32[:, 1] + e32[:, 2], e64[:, 1] + e64[:, 2]
        energy = float(np.abs(tot32 - tot64).max() / np.abs(tot64).max())
        assert energy <= energy_bound, energy
