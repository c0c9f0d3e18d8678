"""CUDA path against the reference on the benchmarked models (fixtures of
tests/golden/timed_models.py: config 2 at its stated geometry and duration,
config 3 at 64 x 64 elements over its 2000 steps, six of the 256 config 4
boreholes over 12,000 steps, the Gaussian and sampled source time functions).

The models are built by the native case builder, whose arrays the CPU test
``test_timed_builder.py`` proves equal to the reference's setup.  Two runs:

* at the reference float build's dt: receiver traces, sample times and (where
  the model records them) wavefield snapshots bit for bit (SHA-256 of all samples; the fixture keeps every k-th row besides, to
  report the size of a difference), the final u, v, a of every domain bit for
  bit (SHA-256 of the float32 fields in the reference's point numbering),
  energy to 1e-9 relative;
* through the timed constructor (the stable dt estimated on the device from
  the arrays it uploads, then the reference's time rule): the same step count
  as the reference for the model's whole duration, dt within 1e-6 relative,
  and receiver traces within 1e-5 relative L2 of the reference float build
  (the bound the backend is held to), measured on the fixture's every k-th
  sample row.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

import golden_io as G
from test_timed_builder import TIMED, timed_fixture, timed_model

pytestmark = pytest.mark.gpu

TRACE_RTOL = 1e-5


def _digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _problem(pkg, case):
    from insem_b200 import cases as K

    z = timed_fixture(case)
    model, _, _ = timed_model(case)
    arrays = K.setup_arrays(model)
    return z, model, arrays


def _check_snapshots(s, z, case):
    """Device snapshots against the reference's (Solver::record_snapshot): same
    times, and every recorded (medium, quantity) field bit for bit."""
    assert np.array_equal(s.snapshot_times, z["snap.times"]), case
    keys = [k[len("hash.snap."):] for k in z.files if k.startswith("hash.snap.")]
    assert keys
    for key in keys:
        medium, quantity = key.split(".")
        got = np.ascontiguousarray(s.snapshot(medium, quantity))
        assert list(got.shape) == list(z[f"shape.snap.{key}"]), (case, key)
        norm = np.linalg.norm(got.astype(np.float64))
        assert _digest(got) == str(z[f"hash.snap.{key}"]), \
            f"{case} {key}: norm {norm:.9e} vs {float(z[f'norm.snap.{key}']):.9e}"


@pytest.mark.parametrize("case", TIMED)
def test_reference_dt_run_bitwise(pkg, case):
    from insem_b200 import cases as K

    z, model, arrays = _problem(pkg, case)
    n_run = int(z["meta.n_steps_run"])
    prob = K.build_from_arrays(model, arrays, stable_dt=float(z["meta.stable_dt"]))
    prob.dt = float(z["meta.dt"])
    prob.n_steps = n_run
    with pkg.Solver(prob) as s:
        if model.snapshot_every > 0:
            s.set_snapshots(model.snapshot_every, model.snapshot_quantities)
        s.advance(n_run // 3)
        s.run()
        assert s.step == n_run
        if model.snapshot_every > 0:
            _check_snapshots(s, z, case)
        stride = int(z["meta.trace_stride"])
        assert _digest(s.times) == str(z["hash.run.times"])
        for name, q in prob.trace_list():
            key = f"run.trace.{name}.{q}"
            got = s.trace(name, q)
            assert list(got.shape) == list(z[f"shape.{key}"])
            err = G.rel_l2(got[::stride], z[key])
            assert _digest(got) == str(z[f"hash.{key}"]), f"{case} {name}/{q}: rel L2 {err:.3e} (every {stride}th row)"
        for di in range(len(prob.domains)):
            for key, arr in zip(("u", "v", "a"), s.state(prob.media[di])):
                f32 = np.ascontiguousarray(arr.astype(np.float32))
                got = _digest(f32)
                norm = np.linalg.norm(f32.astype(np.float64))
                assert got == str(z[f"hash.run.d{di}.{key}"]), \
                    f"{case} d{di} {key}: norm {norm:.9e} vs {float(z[f'norm.run.d{di}.{key}']):.9e}"
        e, ge = s.energy, z["run.energy"]
        assert e.shape == ge.shape
        if ge.size:
            assert np.array_equal(e[:, 0], ge[:, 0])
            scale = np.abs(ge[:, 1:]).max()
            assert np.abs(e[:, 1:] - ge[:, 1:]).max() <= 1e-9 * scale


@pytest.mark.parametrize("case", TIMED)
def test_device_dt_run_within_tolerance(pkg, case):
    from insem_b200 import cases as K

    z, model, arrays = _problem(pkg, case)
    n_run = int(z["meta.n_steps_run"])
    prob, s = K.build_solver_from_arrays(model, arrays)
    with s:
        assert s.n_steps == int(z["meta.n_steps_full"]), (s.n_steps, int(z["meta.n_steps_full"]))
        ref_dt = float(z["meta.dt"])
        assert abs(s.dt - ref_dt) <= 1e-6 * ref_dt, (s.dt, ref_dt)
        s.advance(n_run)
        stride = int(z["meta.trace_stride"])
        worst = 0.0
        for name, q in prob.trace_list():
            key = f"run.trace.{name}.{q}"
            got = s.trace(name, q)
            assert list(got.shape) == list(z[f"shape.{key}"])
            err = G.rel_l2(got[::stride], z[key])
            worst = max(worst, err)
            assert err <= TRACE_RTOL, f"{case} {name}/{q}: rel L2 {err:.3e}"
        print(f"{case}: dt rel diff {abs(s.dt - ref_dt) / ref_dt:.2e}, worst trace rel L2 {worst:.2e}")
