"""The native case builder against the reference's own setup (CPU only).

Each model here describes the same case as tests/golden/cases.py does through
the reference API; every per-step array the builder produces must equal the
array the reference solver built (integers exactly; floats bit for bit).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden


def models(K):
    MUD, STEEL, CEMENT, FAST = K.MUD, K.STEEL, K.CEMENT, K.FAST
    out = {"c1": K.config1()}

    def bh(m_order):
        b = K.borehole((-0.4, 0.64), [("mud", 0.1), ("casing", 0.11), ("cement", 0.14)], formation_radius=1.4,
                       dz=0.08)
        mats = {b.regions["mud"]: MUD, b.regions["casing"]: STEEL, b.regions["cement"]: CEMENT,
                b.regions["formation"]: FAST}
        if m_order == 0:
            src = [K.Source("monopole", 0.0, 0.0, stf=K.ricker(8000.0))]
            rec = [K.Receiver("p1", 0.05, 0.2, ["pressure", "particle_velocity"]),
                   K.Receiver("p2", 0.05, 0.35, ["pressure"]),
                   K.Receiver("s1", 0.3, 0.3, ["velocity", "displacement", "acceleration"])]
        else:
            src = [K.Source("dipole", 0.0, 0.0, (1.0, 0.0, 0.0), K.ricker(3000.0))]
            rec = [K.Receiver("p1", 0.05, 0.2, ["pressure", "particle_velocity"]),
                   K.Receiver("s1", 0.3, 0.3, ["velocity", "displacement"])]
        return K.Model(b.mesh, order=4, f_max=7500.0, azimuthal_order=m_order, materials=mats,
                       boundaries={b.boundaries[n]: "absorbing" for n in ("bottom", "outer", "top")},
                       sources=src, receivers=rec, n_steps=400, energy_every=50, record_every=2)

    out["bh0"], out["bh1"] = bh(0), bh(1)
    interfaces = [-34.0, lambda x: -20.0 + 2.0 * np.sin(2 * np.pi * x / 20.0), 0.0, 6.0]
    m = K.layered((0.0, 40.0), interfaces, [3, 4, 2], [2, 1, 0], nx=12, quadratic=True)
    out["lay"] = K.Model(
        m, order=5,
        materials={0: K.Material.acoustic(1500.0, 1000.0), 1: K.Material.elastic(3000.0, 1600.0, 2200.0),
                   2: K.Material.elastic(4000.0, 2200.0, 2500.0)},
        boundaries={K.BOTTOM: "absorbing", K.RIGHT: "absorbing", K.LEFT: "absorbing", K.TOP: "free"},
        sources=[K.Source("force", 20.0, -6.0, (0.0, 1.0, 0.0), K.ricker(60.0)),
                 K.Source("moment_tensor", 12.0, -25.0, (1.0, 1.0, 0.3), ("gaussian_derivative", 40.0, -1.0, 1.0))],
        receivers=[K.Receiver(f"sf{i}", x, -0.5, ["velocity"], "elastic") for i, x in enumerate((5.0, 15.0, 25.0, 35.0))]
        + [K.Receiver("w0", 10.0, 3.0, ["pressure", "particle_velocity"])],
        n_steps=300, energy_every=25)
    # sheared 6x5 grid, x += 0.3 z, refined region -> affine elements with hanging faces
    nx, nz = 6, 5
    nodes = np.array([(3.0 * i / nx + 0.3 * (2.5 * j / nz), 2.5 * j / nz) for j in range(nz + 1) for i in range(nx + 1)])
    cells, bnd = [], []
    for j in range(nz):
        for i in range(nx):
            c = len(cells)
            n0 = i + (nx + 1) * j
            cells.append([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1])
            for cond, f, t in ((j == 0, 0, 1), (i == nx - 1, 1, 2), (j == nz - 1, 2, 3), (i == 0, 3, 4)):
                if cond:
                    bnd.append((c, f, t))
    mesh = K.MacroMesh(False, False, nodes, np.array(cells, np.int32), np.zeros(len(cells), np.int32),
                       np.array(bnd, np.int32))
    out["box"] = K.Model(mesh, order=3, regions=[(1.0, 2.5, 0.8, 1.6, 1)],
                         materials={0: K.Material.elastic(3000.0, 1700.0, 2000.0)},
                         boundaries={t: "rigid" for t in (1, 2, 3, 4)},
                         receivers=[K.Receiver("c", 1.9, 1.2, ["displacement", "velocity"])],
                         n_steps=200, energy_every=10)
    return out


@pytest.mark.parametrize("case", ["c1", "bh0", "bh1", "lay", "box"])
def test_builder_matches_reference_setup(pkg, case):
    from insem_b200 import cases as K

    z = golden(case)
    arrays = K.setup_arrays(models(K)[case])
    checked = 0
    for key in z.files:
        if not key.startswith("problem.") or key in ("problem.dt", "problem.stable_dt", "problem.n_steps",
                                                     "problem.real_bytes"):
            continue
        if key.endswith((".name", ".quantities", "trace_index")) or key.endswith(".coords"):
            continue
        if key not in arrays and np.asarray(z[key]).size == 0:
            continue  # an empty list (e.g. no sources) stored as an empty array
        assert key in arrays, key
        g, v = np.asarray(z[key]), np.asarray(arrays[key])
        assert v.size == g.size, (key, v.size, g.size)
        v = v.reshape(g.shape).astype(g.dtype)
        if g.dtype.kind == "f":
            assert np.array_equal(v.view(np.uint32 if g.dtype == np.float32 else np.uint64),
                                  g.view(np.uint32 if g.dtype == np.float32 else np.uint64)), key
        else:
            assert np.array_equal(v, g), key
        checked += 1
    assert checked > 20


def test_builder_rejects_bad_models(pkg):
    from insem_b200 import cases as K

    m = K.config1()
    m.materials = {}
    with pytest.raises(K.N.InsemError, match="no material"):
        K.setup_arrays(m)
    m = K.config1()
    m.sources = [K.Source("monopole", 10.0, 10.0, stf=K.ricker(400.0))]
    with pytest.raises(K.N.InsemError, match="not inside"):
        K.setup_arrays(m)


def test_config3_small_shapes(pkg):
    """The benchmark model at 1/16 of its width: two domains, water Rect, elastic Curved."""
    from insem_b200 import cases as K

    m = K.config3(nx=64, n_receivers=16)
    a = K.setup_arrays(m)
    assert int(a["problem.domains.count"][0]) == 2
    kinds = [int(a[f"problem.domains.0.blocks.{b}.kind"][0]) for b in range(int(a["problem.domains.0.blocks.count"][0]))]
    assert kinds == [0]  # water: Rect only
    kinds = [int(a[f"problem.domains.1.blocks.{b}.kind"][0]) for b in range(int(a["problem.domains.1.blocks.count"][0]))]
    assert 2 in kinds
    ng_w, ng_s = int(a["problem.domains.0.n_global"][0]), int(a["problem.domains.1.n_global"][0])
    assert ng_w == (64 * 5 + 1) * (10 * 5 + 1)
    assert ng_s == (64 * 5 + 1) * (54 * 5 + 1)
    assert a["problem.coupling.fluid_points"].size == 64 * 5 + 1
