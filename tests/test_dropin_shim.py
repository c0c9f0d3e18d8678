"""The INSEM_ENABLE_CUDA drop-in shim, end to end (oracle/ref/cuda_shim.cpp).

The shim is compiled against the reference's own sources (test-only target
of oracle/ref/Makefile).  A case is described to the reference's C++
``Simulation`` from this package's macro mesh and model, the reference sets it
up on the CPU (forest, geometry, DofMap, Solver with its stable time step),
and the shim's ``cuda_create`` hands the reference Solver's own arrays to
libinsem_cuda.so through the C ABI; the time loop runs on the GPU and the
results land in the reference Solver's storage.  The traces must equal the
golden fixtures (the reference float build on the CPU) bit for bit.

``run_cpu`` (CPU only) checks the shim's case construction itself: the same
case through the reference's CPU time loop reproduces the fixtures.
"""

from __future__ import annotations

import sys

import numpy as np
import pytest

from conftest import REPO, golden

SHIM_DIR = REPO / "oracle" / "_ref" / "float"
CASES = ["c1", "bh0", "lay"]


def shim():
    if not any(SHIM_DIR.glob("_cudashim*.so")):
        pytest.skip("the reference's oracle build (oracle/_ref) is not present")
    sys.path.insert(0, str(SHIM_DIR))
    import _cudashim

    return _cudashim


def describe(model):
    """A package Model as the shim's arguments (the reference's description)."""
    m = model.mesh
    mesh = dict(nodes=m.nodes, cells=m.cells, region=m.region, boundary=m.boundary, quad9=bool(m.quad9),
                axisymmetric=bool(m.axisymmetric))
    disc = dict(order=model.order, uniform_level=model.uniform_level, f_max=model.f_max,
                points_per_wavelength=model.points_per_wavelength, max_level=model.max_level,
                azimuthal_order=model.azimuthal_order, regions=[list(r) for r in model.regions])
    mats = [(r, x.medium, x.vp, x.vs, x.rho) for r, x in sorted(model.materials.items())]
    bcs = [(t, b) for t, b in sorted(model.boundaries.items())]
    srcs = []
    for s in model.sources:
        st = s.stf
        stf = dict(kind=st[0], f0=st[1], t0=st[2] if st[2] >= 0 or st[0] == "samples" else 1.2 / st[1], amplitude=st[3])
        if st[0] == "samples":
            stf.update(samples=list(st[4]), sample_dt=st[5])
        srcs.append(dict(kind=s.kind, x=s.x, z=s.z, components=list(s.components), stf=stf))
    recs = [dict(name=r.name, x=r.x, z=r.z, quantities=list(r.quantities), medium=r.medium) for r in model.receivers]
    time = dict(n_steps=model.n_steps, duration=model.duration, dt=model.dt, safety=model.safety,
                record_every=model.record_every, energy_every=model.energy_every)
    return mesh, disc, mats, bcs, srcs, recs, time


def model_of(case):
    from insem_b200 import cases as K
    from test_case_builder import models

    return models(K)[case]


def check_results(res, z, case):
    assert np.array_equal(res["times"], z["run.times"]), case
    for key in (k for k in z.files if k.startswith("run.trace.")):
        gold = z[key]
        got = res["traces"][key[len("run.trace."):]]
        assert got.shape == gold.shape, (case, key)
        assert np.array_equal(got, gold), (case, key, float(np.abs(got - gold).max()))
    ge = z["run.energy"]
    assert res["energy"].shape == ge.shape
    if ge.size:
        assert np.array_equal(res["energy"][:, 0], ge[:, 0])
        scale = np.abs(ge[:, 1:]).max()
        assert np.abs(res["energy"][:, 1:] - ge[:, 1:]).max() <= 1e-9 * scale


@pytest.mark.parametrize("case", ["c1", "lay"])
def test_shim_case_reproduces_the_reference_on_the_cpu(pkg, case):
    z = golden(case)
    res = shim().case(*describe(model_of(case))).run_cpu(int(z["run.advance_first"]))
    assert res["dt"] == float(z["problem.dt"]) and res["n_steps"] == int(z["problem.n_steps"])
    check_results(res, z, case)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_reference_simulation_runs_on_the_backend_bitwise(pkg, case):
    z = golden(case)
    res = shim().case(*describe(model_of(case))).run_cuda(int(z["run.advance_first"]))
    assert res["step"] == int(z["problem.n_steps"])
    check_results(res, z, case)
