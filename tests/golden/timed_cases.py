"""The benchmarked configurations through the reference's own Python API.

Test infrastructure only: imported by ``make_golden.py --timed`` with the
reference package (``insem``, built by ``oracle/ref/Makefile``) on
``sys.path``.  For every model of ``timed_models.py`` it builds the macro mesh
with the reference's template named in the model's recipe and describes the
same model through the reference's ``Simulation``, so that the fixtures hold
the reference's own setup and results for the models that this package times.
"""

from __future__ import annotations

import insem
from insem import mesh

import timed_models


def _ref_material(m):
    if m.medium == "acoustic":
        return insem.Material.acoustic(m.vp, m.rho)
    return insem.Material.elastic(m.vp, m.vs, m.rho)


def _ref_stf(stf):
    kind = stf[0]
    if kind == "samples":
        return insem.sampled_stf(stf[4], stf[5], stf[3])
    f = {"ricker": insem.ricker, "gaussian": insem.gaussian, "gaussian_derivative": insem.gaussian_derivative}[kind]
    return f(stf[1], None if stf[2] < 0 else stf[2], stf[3])


def _ref_source(s):
    stf = _ref_stf(s.stf)
    c = s.components
    if s.kind == "monopole":
        return insem.Source.monopole(s.x, s.z, stf)
    if s.kind == "dipole":
        return insem.Source.dipole(s.x, s.z, c[0], c[1], stf)
    if s.kind == "force":
        return insem.Source.force(s.x, s.z, c[0], c[1], stf)
    return insem.Source.moment_tensor(s.x, s.z, c[0], c[1], c[2], stf)


def ref_mesh(recipe):
    name, args, kw = recipe
    m = getattr(mesh, name)(*args, **kw)
    return m.mesh if hasattr(m, "regions") and hasattr(m, "mesh") else m


def ref_simulation(model, recipe):
    """The reference Simulation of a package Model, on the reference-built macro mesh."""
    disc = insem.Discretization(order=model.order, uniform_level=model.uniform_level, f_max=model.f_max,
                                points_per_wavelength=model.points_per_wavelength, max_level=model.max_level,
                                regions=[tuple(r) for r in model.regions], azimuthal_order=model.azimuthal_order)
    sim = insem.Simulation(ref_mesh(recipe), disc)
    for region, m in model.materials.items():
        sim.set_material(region, _ref_material(m))
    for tag, bc in model.boundaries.items():
        sim.set_boundary(tag, bc)
    for s in model.sources:
        sim.add_source(_ref_source(s))
    for r in model.receivers:
        if r.medium:
            sim.add_receiver(r.name, r.x, r.z, list(r.quantities), r.medium)
        else:
            sim.add_receiver(r.name, r.x, r.z, list(r.quantities))
    sim.set_time(n_steps=model.n_steps, duration=model.duration, dt=model.dt, safety=model.safety,
                 record_every=model.record_every, energy_every=model.energy_every,
                 snapshot_every=model.snapshot_every, snapshot_quantities=list(model.snapshot_quantities))
    return sim


def _case(make):
    def build():
        model, n_run, recipe = make()
        return ref_simulation(model, recipe), n_run, model
    return build


TIMED_CASES = {name: _case(make) for name, make in timed_models.TIMED.items()}
