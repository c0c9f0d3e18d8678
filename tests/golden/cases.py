"""Cases for the golden fixtures, written against the reference's own Python API.

Test infrastructure only: imported by ``make_golden.py`` with the reference
package (``insem``, built by ``oracle/ref/Makefile``) on ``sys.path``.  Each
builder returns ``(simulation, init)`` where ``init`` optionally sets an
initial state on the reference solver before its first step.

The cases cover every kernel variant and boundary treatment on the per-step
path at sizes the CPU finishes in seconds:

* ``c1``   -- the README example (2D Cartesian acoustic, 32x32 quads, order 4,
  Stacey on all sides, Ricker 400 Hz monopole, pressure receiver at (1.5, 0),
  4 ms), i.e. the reference's plain CPU-runnable case.
* ``bh0``  -- a short cased borehole, azimuthal order 0, AMR with hanging
  faces, fluid-solid coupling, Stacey on bottom/outer/top, symmetry axis.
* ``bh1``  -- the same borehole at azimuthal order 1 (dipole source).
* ``lay``  -- 2D Cartesian coupled water over two curved elastic layers
  (Quad9 cells, order 5), free surface on top, Stacey elsewhere.
* ``box``  -- sheared (affine) elastic box with rigid walls, a refined
  region (hanging faces in Cartesian mode) and an initial Gaussian pulse set
  through ``set_state``; no source; the energy monitor is on.
* ``blk<N>`` -- tiny meshes per number of GLL points N = 2..9 (orders 1..8)
  covering Rect, Affine, Curved and Axisym m = 0 / m = 1 blocks, acoustic and
  elastic, for per-block force vectors only.
"""

from __future__ import annotations

import numpy as np

import insem
from insem import mesh

MUD = insem.Material.acoustic(1500.0, 1000.0)
STEEL = insem.Material.elastic(5900.0, 3200.0, 7850.0)
CEMENT = insem.Material.elastic(3000.0, 1600.0, 1900.0)
FAST = insem.Material.elastic(4000.0, 2300.0, 2400.0)
WATER = insem.Material.acoustic(1500.0, 1000.0)


def sheared_grid(nx, nz, x0, x1, z0, z1, shear, material=None, coords="cartesian"):
    """Quad4 grid with x += shear * z (parallelogram cells), tags 1..4 = bottom/right/top/left."""
    nodes = []
    for j in range(nz + 1):
        for i in range(nx + 1):
            z = z0 + (z1 - z0) * j / nz
            nodes.append((x0 + (x1 - x0) * i / nx + shear * z, z))
    cells, mat, bnd = [], [], []
    for j in range(nz):
        for i in range(nx):
            c = len(cells)
            n0 = i + (nx + 1) * j
            cells.append([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1])
            mat.append(0 if material is None else material(i, j))
            if j == 0:
                bnd.append((c, 0, 1))
            if i == nx - 1:
                bnd.append((c, 1, 2))
            if j == nz - 1:
                bnd.append((c, 2, 3))
            if i == 0:
                bnd.append((c, 3, 4))
    return insem.MacroMesh("quad4", coords, np.asarray(nodes, float), np.asarray(cells, np.int32),
                           np.asarray(mat, np.int32), np.asarray(bnd, np.int32).reshape(-1, 3))


def c1():
    m = mesh.rectangle((-4.0, 4.0), (-4.0, 4.0), nx=32, nz=32)
    sim = insem.Simulation(m, insem.Discretization(order=4))
    sim.set_material(0, insem.Material.acoustic(vp=1500.0, rho=1000.0))
    for tag in (mesh.BOTTOM, mesh.RIGHT, mesh.TOP, mesh.LEFT):
        sim.set_boundary(tag, "absorbing")
    sim.add_source(insem.Source.monopole(0.0, 0.0, insem.ricker(400.0)))
    sim.add_receiver("h1", 1.5, 0.0, ["pressure"])
    sim.set_time(duration=4e-3)
    return sim, None


def _borehole(m_order: int):
    b = mesh.borehole((-0.4, 0.64), [("mud", 0.1), ("casing", 0.11), ("cement", 0.14)],
                      formation_radius=1.4, dz=0.08)
    sim = insem.Simulation(b.mesh, insem.Discretization(order=4, f_max=7500.0, azimuthal_order=m_order))
    for name, mat in (("mud", MUD), ("casing", STEEL), ("cement", CEMENT), ("formation", FAST)):
        sim.set_material(b.regions[name], mat)
    for name in ("bottom", "outer", "top"):
        sim.set_boundary(b.boundaries[name], "absorbing")
    if m_order == 0:
        sim.add_source(insem.Source.monopole(0.0, 0.0, insem.ricker(8000.0)))
        sim.add_receiver("p1", 0.05, 0.2, ["pressure", "particle_velocity"])
        sim.add_receiver("p2", 0.05, 0.35, ["pressure"])
        sim.add_receiver("s1", 0.3, 0.3, ["velocity", "displacement", "acceleration"])
    else:
        sim.add_source(insem.Source.dipole(0.0, 0.0, 1.0, 0.0, insem.ricker(3000.0)))
        sim.add_receiver("p1", 0.05, 0.2, ["pressure", "particle_velocity"])
        sim.add_receiver("s1", 0.3, 0.3, ["velocity", "displacement"])
    sim.set_time(n_steps=400, energy_every=50, record_every=2)
    return sim, None


def bh0():
    return _borehole(0)


def bh1():
    return _borehole(1)


def lay():
    interfaces = [-34.0, lambda x: -20.0 + 2.0 * np.sin(2 * np.pi * x / 20.0), 0.0, 6.0]
    m = mesh.layered((0.0, 40.0), interfaces, [3, 4, 2], [2, 1, 0], nx=12, quadratic=True)
    sim = insem.Simulation(m, insem.Discretization(order=5))
    sim.set_material(0, WATER)
    sim.set_material(1, insem.Material.elastic(3000.0, 1600.0, 2200.0))
    sim.set_material(2, insem.Material.elastic(4000.0, 2200.0, 2500.0))
    for tag in (mesh.BOTTOM, mesh.RIGHT, mesh.LEFT):
        sim.set_boundary(tag, "absorbing")
    sim.set_boundary(mesh.TOP, "free")
    sim.add_source(insem.Source.force(20.0, -6.0, 0.0, 1.0, insem.ricker(60.0)))
    sim.add_source(insem.Source.moment_tensor(12.0, -25.0, 1.0, 1.0, 0.3, insem.gaussian_derivative(40.0)))
    for i, x in enumerate((5.0, 15.0, 25.0, 35.0)):
        sim.add_receiver(f"sf{i}", x, -0.5, ["velocity"], "elastic")
    sim.add_receiver("w0", 10.0, 3.0, ["pressure", "particle_velocity"])
    sim.set_time(n_steps=300, energy_every=25)
    return sim, None


def box():
    m = sheared_grid(6, 5, 0.0, 3.0, 0.0, 2.5, 0.3)
    sim = insem.Simulation(m, insem.Discretization(order=3, regions=[(1.0, 2.5, 0.8, 1.6, 1)]))
    sim.set_material(0, insem.Material.elastic(3000.0, 1700.0, 2000.0))
    for tag in (1, 2, 3, 4):
        sim.set_boundary(tag, "rigid")
    sim.add_receiver("c", 1.9, 1.2, ["displacement", "velocity"])
    sim.set_time(n_steps=200, energy_every=10)

    def init(solver):
        xz = solver.coordinates("elastic")
        r2 = (xz[0] - 1.9) ** 2 + (xz[1] - 1.2) ** 2
        g = np.exp(-r2 / 0.08)
        u = np.stack([g, 0.5 * g])
        v = np.stack([0.0 * g, 20.0 * g])
        solver.set_state("elastic", u, v)

    return sim, init


def blk(ngll: int):
    """Tiny meshes covering every block kind for one GLL point count (no time loop)."""
    order = ngll - 1
    sims = []
    # Rect + Affine, acoustic and elastic (two media side by side -> coupling too).
    for shear in (0.0, 0.35):
        m = sheared_grid(4, 2, 0.0, 2.0, 0.0, 1.0, shear, material=lambda i, j: 0 if i < 2 else 1)
        sim = insem.Simulation(m, insem.Discretization(order=order))
        sim.set_material(0, insem.Material.acoustic(1500.0, 1000.0))
        sim.set_material(1, insem.Material.elastic(3000.0, 1700.0, 2000.0))
        sims.append(sim)
    # Curved (Quad9 layered), acoustic over elastic.
    m = mesh.layered((0.0, 2.0), [-1.0, lambda x: 0.1 * np.sin(3.0 * x), 0.6], 1, [1, 0], nx=3, quadratic=True)
    sim = insem.Simulation(m, insem.Discretization(order=order))
    sim.set_material(0, insem.Material.acoustic(1500.0, 1000.0))
    sim.set_material(1, insem.Material.elastic(3000.0, 1700.0, 2000.0))
    sims.append(sim)
    # Axisymmetric, azimuthal orders 0 and 1: a mud column on the axis (axial
    # acoustic, non-axial elastic) and an elastic column on the axis (axial
    # elastic, non-axial acoustic).
    for m_order in (0, 1):
        b = mesh.borehole((0.0, 0.3), [("mud", 0.1)], formation_radius=0.35, dz=0.1, dr=0.12)
        sim = insem.Simulation(b.mesh, insem.Discretization(order=order, azimuthal_order=m_order))
        sim.set_material(b.regions["mud"], MUD)
        sim.set_material(b.regions["formation"], FAST)
        sims.append(sim)
        m = mesh.rectangle((0.0, 0.2, 0.45), (0.0, 0.15, 0.3), material=lambda x, z: 1 if x < 0.2 else 0,
                           coords="axisymmetric")
        sim = insem.Simulation(m, insem.Discretization(order=order, azimuthal_order=m_order))
        sim.set_material(0, MUD)
        sim.set_material(1, FAST)
        sims.append(sim)
    for sim in sims:
        sim.set_time(n_steps=1)
    return sims


RUN_CASES = {"c1": c1, "bh0": bh0, "bh1": bh1, "lay": lay, "box": box}
