"""The benchmarked configurations as this package's models, for the timed-config fixtures.

Test infrastructure only.  Each function returns ``(model, n_run, recipe)``:

* ``model``  -- the ``insem_b200.cases.Model`` that ``bench.py`` and the server
  build (the same workload functions, seeds and shipped geometry table);
* ``n_run``  -- steps the fixture runs (0: the model's whole duration);
* ``recipe`` -- ``(template, args, kwargs)`` of the macro mesh, so that the
  fixture generator (``timed_cases.py``) builds the same mesh with the
  reference's own template of that name and feeds it to the reference's
  setup.  The builder test then proves the two setups give identical arrays.

Cases:

* ``c2``   -- the cased borehole of config 2 at its stated geometry
  (z in [-1.5, 4.5] m, formation radius 4 m, dz 0.08, order 4, f_max 7.5 kHz,
  13 pressure receivers at r = 0.05 m, z = 2.0 ... 3.8 m), the full 5 ms.
* ``c3s``  -- config 3's coupled water / 8 curved layers model at 64 x 64
  elements, order 5, its 2000 steps, 16 seafloor receivers.
* ``c4m<k>`` -- model k of config 4's 256 seeded boreholes with its shipped
  geometry; 12,000 steps (the 13 receivers at z >= 2 m see the direct waves),
  or the model's whole duration if shorter.  The set spans m = 0 / 1,
  GLL orders 4, 5 and 6 (NG 5, 6, 7), cased and uncased holes and slow
  formations (vs < 1500 m/s).
* ``stfg`` -- a small coupled Cartesian model driven by Gaussian source time
  functions (a force and a monopole).
* ``stfs`` -- a small acoustic model driven by a sampled source time function
  whose samples end inside the run (dt = 2^-17 s, sample interval 2^-16 s, so
  one step lands exactly on the last sample).

Every case records the energy monitor, so the fixtures also carry the energy
of the float and the double build.
"""

from __future__ import annotations

import numpy as np

import __graft_entry__ as entry

entry.load_package()
from insem_b200 import cases as K  # noqa: E402

C4_MODELS = (0, 1, 12, 17, 72, 80)
C4_STEPS = 12000
ENERGY_EVERY = 100


def c2():
    model = K.config2()
    model.energy_every = ENERGY_EVERY
    recipe = ("borehole", ((-1.5, 4.5), [("mud", 0.1), ("casing", 0.11), ("cement", 0.14)]),
              dict(formation_radius=4.0, dz=0.08))
    return model, 0, recipe


def c3s():
    nx = 64
    model = K.config3(nx=nx, n_steps=2000, n_receivers=16)
    model.energy_every = ENERGY_EVERY
    spec = K.config3_spec(nx, 3, 16)
    recipe = ("layered", ((0.0, 400.0), spec["interfaces"], spec["counts"], spec["regions"]),
              dict(nx=nx, quadratic=True))
    return model, 0, recipe


def c4(index: int):
    params = K.config4_params(256, 4)[index]
    zlen, radius = K.config4_geometry_table(256, 4)[index]
    model = K.config4_model(params, zlen, radius)
    model.energy_every = ENERGY_EVERY
    hole = params["hole"]
    ann = [("mud", hole)] + ([("casing", hole + 0.01), ("cement", hole + 0.04)] if params["casing"] else [])
    z0 = -1.5
    beds = [(z0, "bed0")] + [(z0 + zlen * f, f"bed{i + 1}") for i, f in enumerate(params["bed_fracs"])]
    recipe = ("borehole", ((z0, z0 + zlen), ann), dict(formation_radius=radius, beds=beds, dz=0.08))
    return model, C4_STEPS, recipe


def stfg():
    interfaces = [-12.0, lambda x: -5.0 + 0.8 * np.sin(2 * np.pi * x / 9.0), 0.0, 4.0]
    args, kw = ((0.0, 16.0), interfaces, [3, 2, 2], [1, 2, 0]), dict(nx=8, quadratic=True)
    model = K.Model(
        K.layered(*args, **kw), order=4,
        materials={0: K.Material.acoustic(1500.0, 1000.0), 1: K.Material.elastic(3200.0, 1800.0, 2300.0),
                   2: K.Material.elastic(2600.0, 1300.0, 2100.0)},
        boundaries={K.BOTTOM: "absorbing", K.RIGHT: "absorbing", K.LEFT: "absorbing", K.TOP: "free"},
        sources=[K.Source("force", 6.0, -3.0, (0.3, 1.0, 0.0), K.gaussian(150.0)),
                 K.Source("monopole", 10.0, 1.5, stf=K.gaussian(120.0, 0.011, 2.5))],
        receivers=[K.Receiver("s0", 3.0, -1.0, ["velocity", "displacement"], "elastic"),
                   K.Receiver("s1", 12.5, -8.0, ["acceleration"]),
                   K.Receiver("w0", 8.0, 2.0, ["pressure", "particle_velocity"])],
        n_steps=500, energy_every=25)
    return model, 0, ("layered", args, kw)


def stfs():
    t = np.arange(160) * 2.0 ** -16
    samples = np.sin(2 * np.pi * 350.0 * t) * np.exp(-((t - 1.2e-3) / 6e-4) ** 2)
    args, kw = ((-4.0, 4.0), (-3.0, 3.0)), dict(nx=16, nz=12)
    model = K.Model(
        K.rectangle(*args, **kw), order=4, materials={0: K.Material.acoustic(1500.0, 1000.0)},
        boundaries={K.BOTTOM: "absorbing", K.RIGHT: "absorbing", K.TOP: "free", K.LEFT: "rigid"},
        sources=[K.Source("monopole", 0.3, -0.2, stf=K.sampled(samples, 2.0 ** -16, 1.5))],
        receivers=[K.Receiver("h0", 1.5, 0.5, ["pressure", "particle_velocity"]),
                   K.Receiver("h1", -2.0, -1.0, ["pressure"])],
        n_steps=400, dt=2.0 ** -17, energy_every=20)
    return model, 0, ("rectangle", args, kw)


def snapbh1():
    """A short cased borehole at azimuthal order 1 (hanging faces, fluid-solid
    coupling, the axis) recording wavefield snapshots of every quantity."""
    b = K.borehole((-0.4, 0.64), [("mud", 0.1), ("casing", 0.11), ("cement", 0.14)], formation_radius=1.4, dz=0.08)
    recipe = ("borehole", ((-0.4, 0.64), [("mud", 0.1), ("casing", 0.11), ("cement", 0.14)]),
              dict(formation_radius=1.4, dz=0.08))
    mats = {b.regions["mud"]: K.MUD, b.regions["casing"]: K.STEEL, b.regions["cement"]: K.CEMENT,
            b.regions["formation"]: K.FAST}
    model = K.Model(b.mesh, order=4, f_max=7500.0, azimuthal_order=1, materials=mats,
                    boundaries={b.boundaries[n]: "absorbing" for n in ("bottom", "outer", "top")},
                    sources=[K.Source("dipole", 0.0, 0.0, (1.0, 0.0, 0.0), K.ricker(3000.0))],
                    receivers=[K.Receiver("p1", 0.05, 0.2, ["pressure"])], n_steps=240,
                    snapshot_every=60, snapshot_quantities=("velocity", "pressure", "displacement", "acceleration"))
    return model, 0, recipe


def snaplay():
    """Water over two curved elastic layers (Quad9 cells) recording velocity
    and pressure snapshots, with a refined region (hanging faces)."""
    interfaces = [-12.0, lambda x: -5.0 + 0.8 * np.sin(2 * np.pi * x / 9.0), 0.0, 4.0]
    args, kw = ((0.0, 16.0), interfaces, [3, 2, 2], [1, 2, 0]), dict(nx=8, quadratic=True)
    model = K.Model(
        K.layered(*args, **kw), order=4, regions=[(4.0, 9.0, -8.0, -2.0, 1)],
        materials={0: K.Material.acoustic(1500.0, 1000.0), 1: K.Material.elastic(3200.0, 1800.0, 2300.0),
                   2: K.Material.elastic(2600.0, 1300.0, 2100.0)},
        boundaries={K.BOTTOM: "absorbing", K.RIGHT: "absorbing", K.LEFT: "absorbing", K.TOP: "free"},
        sources=[K.Source("force", 6.0, -3.0, (0.3, 1.0, 0.0), K.ricker(150.0))],
        receivers=[K.Receiver("w0", 8.0, 2.0, ["pressure"])], n_steps=300, snapshot_every=75)
    return model, 0, ("layered", args, kw)


TIMED = {"c2": c2, "c3s": c3s, "stfg": stfg, "stfs": stfs, "snapbh1": snapbh1, "snaplay": snaplay}
TIMED.update({f"c4m{k}": (lambda k=k: c4(k)) for k in C4_MODELS})
