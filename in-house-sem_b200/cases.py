"""Model descriptions and the benchmark / serving workloads, built natively.

``Model`` holds what the reference's ``Simulation`` describes (mesh,
discretisation, materials, boundaries, sources, receivers, time settings,
cpp/include/insem/sim/simulation.hpp:56-124); ``build`` runs the native
setup (csrc/host/cases.cpp) and the device power iteration for the stable
time step, and returns the ``ProblemData`` the solver takes.

The mesh templates (rectangle, layered, borehole) produce the macro meshes
of the reference's templates (python/insem/mesh/templates.py) node for node,
so that a model described here and through the reference set up identically.

Workloads (seeded; shapes and value ranges as the benchmark configurations
state them):
  config1   32x32 acoustic rectangle, order 4, Stacey, Ricker 400 Hz (4 ms)
  config2   cased borehole m = 0, order 4, f_max 7.5 kHz, AMR (5 ms)
  config3   1024x1024 coupled water / 8 curved elastic layers, order 5 (2000 steps)
  config4   256 boreholes, m = 0 / 1, order 4-6, 1-6 beds, casing in 30 %
  serving   Poisson mix of Cartesian and borehole requests
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple, Union

import numpy as np

from . import native as N
from .problem import ProblemData

BOTTOM, RIGHT, TOP, LEFT = 1, 2, 3, 4
MEDIUM = {"acoustic": 0, "elastic": 1}
BC = {"free": 0, "rigid": 1, "absorbing": 2}
SOURCE_KIND = {"force": 0, "moment_tensor": 1, "monopole": 2, "dipole": 3}
STF_KIND = {"ricker": 0, "gaussian": 1, "gaussian_derivative": 2, "samples": 3}


# ------------------------------------------------------------------ meshes
# Structured macro meshes.  Cells are numbered row by row (x fastest), corners
# counter-clockwise from (-1, -1), Quad9 side midpoints then the centre; the
# boundary sides carry the tags BOTTOM 1, RIGHT 2, TOP 3, LEFT 4, listed per
# cell in side order.  These are the conventions of the reference's mesh
# templates (python/insem/mesh/templates.py), whose node coordinates the
# builder tests require bit for bit: breakpoints are np.linspace, Quad9
# midpoints the mean of their two breakpoints, layer rows the linear blend
# (1 - t) z_bottom + t z_top with t = row / rows, radial grading the running
# sum of geometrically growing sizes.
@dataclass
class MacroMesh:
    quad9: bool
    axisymmetric: bool
    nodes: np.ndarray      # (n_nodes, 2)
    cells: np.ndarray      # (n_cells, 4 or 9)
    region: np.ndarray     # (n_cells,)
    boundary: np.ndarray   # (n_faces, 3) cell, face, tag


def _breakpoints(spec, cells: Optional[int]) -> np.ndarray:
    """Either explicit breakpoints, or (lo, hi) split into `cells` equal cells."""
    v = np.asarray(spec, float)
    return v if cells is None else np.linspace(v[0], v[1], cells + 1)


def _node_positions(breaks: np.ndarray, quad9: bool) -> np.ndarray:
    """Node positions along one direction: the breakpoints, and for Quad9 cells
    the midpoint of every interval between them."""
    if not quad9:
        return breaks
    mids = (breaks[:-1] + breaks[1:]) * 0.5
    return np.append(np.column_stack([breaks[:-1], mids]).ravel(), breaks[-1])


_QUAD9_OFFSETS = np.array([(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)])
_QUAD4_OFFSETS = np.array([(0, 0), (1, 0), (1, 1), (0, 1)])


def _grid_mesh(columns: np.ndarray, heights: np.ndarray, quad9: bool, region: np.ndarray, axisym: bool) -> MacroMesh:
    """Macro mesh on a node grid: `columns` (m,) x positions, `heights` (rows, m)
    node z per grid row."""
    stride = 2 if quad9 else 1
    m = columns.size
    ncx, ncz = (m - 1) // stride, (heights.shape[0] - 1) // stride
    if np.any(np.diff(heights, axis=0) <= 0):
        raise ValueError("grid rows must rise strictly in z at every x (zero-thickness layers?)")
    nodes = np.column_stack([np.tile(columns, heights.shape[0]), heights.ravel()])
    c = np.arange(ncx * ncz)
    ci, cj = c % ncx, c // ncx
    off = _QUAD9_OFFSETS if quad9 else _QUAD4_OFFSETS
    cells = (stride * ci[:, None] + off[None, :, 0]) + m * (stride * cj[:, None] + off[None, :, 1])
    # boundary sides: (cell, side, tag), ordered by cell then side
    sides = np.stack([cj == 0, ci == ncx - 1, cj == ncz - 1, ci == 0], axis=1)
    cell_of, side_of = np.nonzero(sides)
    tags = np.array([BOTTOM, RIGHT, TOP, LEFT])[side_of]
    boundary = np.column_stack([cell_of, side_of, tags])
    return MacroMesh(quad9, axisym, np.ascontiguousarray(nodes, float), np.ascontiguousarray(cells, np.int32),
                     np.ascontiguousarray(region, np.int32), np.ascontiguousarray(boundary, np.int32))


def rectangle(x, z, nx=None, nz=None, material: Union[int, Sequence[int], Callable] = 0, quadratic=False,
              coords="cartesian") -> MacroMesh:
    """Rectangle of nx x nz cells (or explicit breakpoints); `material` is a
    region id, one id per cell, or f(x_centre, z_centre) -> id (vectorised when
    the function has ``vectorized = True``)."""
    xb, zb = _breakpoints(x, nx), _breakpoints(z, nz)
    ncx, ncz = xb.size - 1, zb.size - 1
    cols = _node_positions(xb, quadratic)
    rows = np.repeat(_node_positions(zb, quadratic)[:, None], cols.size, axis=1)
    if callable(material):
        xc = np.tile((xb[:-1] + xb[1:]) * 0.5, ncz)
        zc = np.repeat((zb[:-1] + zb[1:]) * 0.5, ncx)
        if getattr(material, "vectorized", False):
            region = np.asarray(material(xc, zc), np.int32)
        else:
            region = np.array([material(a, b) for a, b in zip(xc, zc)], np.int32)
    else:
        region = np.broadcast_to(np.asarray(material, np.int32), (ncx * ncz,)).copy()
    return _grid_mesh(cols, rows, quadratic, region, coords == "axisymmetric")


def layered(x, interfaces, nz, regions, nx=None, quadratic=False, coords="cartesian") -> MacroMesh:
    """Layers between K + 1 interfaces (heights or vectorised z(x)), bottom to
    top, with nz cells across each (one count or K counts) and region ids
    `regions`; node rows inside a layer blend its two interfaces linearly."""
    xb = _breakpoints(x, nx)
    cols = _node_positions(xb, quadratic)
    n_layers = len(interfaces) - 1
    counts = [int(nz)] * n_layers if np.isscalar(nz) else [int(v) for v in nz]
    surfaces = [np.broadcast_to(np.asarray(f(cols) if callable(f) else float(f), float), cols.shape).astype(float)
                for f in interfaces]
    stride = 2 if quadratic else 1
    blocks = [surfaces[0][None, :]]
    for k in range(n_layers):
        steps = stride * counts[k]
        t = (np.arange(1, steps + 1) / steps)[:, None]
        blocks.append((1.0 - t) * surfaces[k][None, :] + t * surfaces[k + 1][None, :])
    region = np.repeat(np.asarray(regions[:n_layers], np.int32), [(xb.size - 1) * c for c in counts])
    return _grid_mesh(cols, np.vstack(blocks), quadratic, region, coords == "axisymmetric")


def _grown_breaks(start: float, stop: float, first: float, growth: float, cap: float) -> List[float]:
    """Breakpoints from start to stop for cells of size first, first * growth,
    ... (at most cap); a remainder shorter than 1.5 cells joins the last one."""
    out = [start]
    size = first
    while stop - out[-1] > 1e-12 * max(1.0, abs(stop)):
        size = min(size, cap)
        if stop - out[-1] <= 1.5 * size:
            out.append(stop)
            break
        out.append(out[-1] + size)
        size *= growth
    return out


@dataclass
class Borehole:
    mesh: MacroMesh
    regions: Dict[str, int]
    boundaries: Dict[str, int]


def borehole(z, annuli, formation_radius, beds=(), dz=0.05, dr=None, growth=1.3, fluid_cells=2,
             quadratic=False) -> Borehole:
    """Axisymmetric (r, z) borehole: `annuli` = [(name, outer radius), ...] from
    the axis out (the fluid column gets `fluid_cells` radial cells, the others
    about one cell per dz), then the formation out to `formation_radius` with
    cells growing by `growth` up to `dr` (default 4 dz), split into `beds` =
    [(z_bottom, name), ...].  Region ids count from 1 in order of first
    appearance, annuli before beds; tags: bottom 1, outer 2, top 3, axis 4."""
    z0, z1 = float(z[0]), float(z[1])
    names = [a for a, _ in annuli]
    outer = [float(r) for _, r in annuli]
    beds = list(beds) or [(z0, "formation")]
    cap = 4 * dz if dr is None else dr

    def cells_across(a: float, b: float) -> int:
        return max(1, int(np.ceil((b - a) / dz - 1e-9)))

    r = list(np.linspace(0.0, outer[0], fluid_cells + 1))
    last_cell = outer[0] / fluid_cells
    for a, b in zip(outer[:-1], outer[1:]):
        k = cells_across(a, b)
        r.extend(np.linspace(a, b, k + 1)[1:])
        last_cell = (b - a) / k
    r.extend(_grown_breaks(outer[-1], formation_radius, min(last_cell * growth, cap), growth, cap)[1:])

    bottoms = [float(b[0]) for b in beds]
    zs = [z0]
    for a, b in zip(bottoms, bottoms[1:] + [z1]):
        zs.extend(np.linspace(a, b, cells_across(a, b) + 1)[1:])

    ids = {name: i + 1 for i, name in enumerate(dict.fromkeys(names + [b[1] for b in beds]))}
    annulus_ids = np.array([ids[n] for n in names], np.int32)
    bed_ids = np.array([ids[b[1]] for b in beds], np.int32)
    outer_arr = np.array(outer)

    def region(rc, zc):
        rc, zc = np.asarray(rc, float), np.asarray(zc, float)
        inside = rc[:, None] < outer_arr[None, :]             # the first annulus whose outer radius exceeds rc
        ring = np.argmax(inside, axis=1)
        bed = bed_ids[np.searchsorted(np.array(bottoms), zc, side="right") - 1]
        return np.where(inside.any(axis=1), annulus_ids[ring], bed)

    region.vectorized = True
    m = rectangle(r, zs, material=region, quadratic=quadratic, coords="axisymmetric")
    return Borehole(m, ids, {"bottom": BOTTOM, "outer": RIGHT, "top": TOP, "axis": LEFT})


# ------------------------------------------------------------------ model
@dataclass
class Material:
    medium: str
    vp: float
    vs: float
    rho: float

    @staticmethod
    def acoustic(vp, rho):
        return Material("acoustic", vp, 0.0, rho)

    @staticmethod
    def elastic(vp, vs, rho):
        return Material("elastic", vp, vs, rho)


@dataclass
class Source:
    kind: str
    x: float
    z: float
    components: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    stf: Tuple[str, float, float, float] = ("ricker", 1.0, -1.0, 1.0)  # kind, f0, t0 (-1: 1.2/f0), amplitude


def ricker(f0, t0=-1.0, amplitude=1.0):
    return ("ricker", f0, t0, amplitude)


def gaussian(f0, t0=-1.0, amplitude=1.0):
    return ("gaussian", f0, t0, amplitude)


def gaussian_derivative(f0, t0=-1.0, amplitude=1.0):
    return ("gaussian_derivative", f0, t0, amplitude)


def sampled(samples, dt, amplitude=1.0):
    """Samples at t = i * dt, linearly interpolated, zero outside [0, (n - 1) dt]."""
    samples = np.asarray(samples, np.float64)
    if dt <= 0.0 or samples.size == 0:
        raise ValueError("a sampled source time function needs samples and a positive interval")
    return ("samples", 0.0, 0.0, amplitude, samples, float(dt))


@dataclass
class Receiver:
    name: str
    x: float
    z: float
    quantities: List[str]
    medium: str = ""


@dataclass
class Model:
    mesh: MacroMesh
    order: int = 4
    uniform_level: int = 0
    f_max: float = 0.0
    points_per_wavelength: float = 5.0
    max_level: int = 12
    regions: List[Tuple[float, float, float, float, int]] = field(default_factory=list)
    azimuthal_order: int = 0
    materials: Dict[int, Material] = field(default_factory=dict)
    boundaries: Dict[int, str] = field(default_factory=dict)
    sources: List[Source] = field(default_factory=list)
    receivers: List[Receiver] = field(default_factory=list)
    duration: float = 0.0
    n_steps: int = 0
    dt: float = 0.0
    safety: float = 0.8
    record_every: int = 1
    energy_every: int = 0
    snapshot_every: int = 0  # wavefield snapshots (Solver.set_snapshots), 0 = off
    snapshot_quantities: Tuple[str, ...] = ("velocity", "pressure")


_cases_lib = None


def cases_lib() -> C.CDLL:
    global _cases_lib
    if _cases_lib is None:
        path = N.PKG / "lib" / "libinsem_cases.so"
        if not path.exists():
            raise N.InsemError(N.ERR_INVALID, f"case setup library missing: {path} (run build.py)")
        L = C.CDLL(str(path))
        L.insem_case_build.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.insem_case_build.restype = C.c_int
        L.insem_case_n_arrays.argtypes = [C.c_void_p]
        L.insem_case_n_arrays.restype = C.c_int32
        L.insem_case_array_at.argtypes = [C.c_void_p, C.c_int32]
        L.insem_case_array_at.restype = C.c_void_p
        L.insem_case_free.argtypes = [C.c_void_p]
        L.insem_case_last_error.restype = C.c_char_p
        _cases_lib = L
    return _cases_lib


class _Desc(C.Structure):
    _fields_ = [("quad9", C.c_int32), ("axisymmetric", C.c_int32), ("n_nodes", C.c_int32), ("nodes", C.c_void_p),
                ("n_cells", C.c_int32), ("cells", C.c_void_p), ("cell_region", C.c_void_p),
                ("n_boundary", C.c_int32), ("boundary", C.c_void_p), ("order", C.c_int32),
                ("uniform_level", C.c_int32), ("f_max", C.c_double), ("points_per_wavelength", C.c_double),
                ("max_level", C.c_int32), ("n_regions", C.c_int32), ("regions", C.c_void_p),
                ("azimuthal_order", C.c_int32), ("n_materials", C.c_int32), ("material_region", C.c_void_p),
                ("material_medium", C.c_void_p), ("material_vp", C.c_void_p), ("material_vs", C.c_void_p),
                ("material_rho", C.c_void_p), ("n_bc", C.c_int32), ("bc_tag", C.c_void_p), ("bc_type", C.c_void_p),
                ("n_sources", C.c_int32), ("source_kind", C.c_void_p), ("source_position", C.c_void_p),
                ("source_components", C.c_void_p), ("stf_kind", C.c_void_p), ("stf_params", C.c_void_p),
                ("n_receivers", C.c_int32), ("receiver_position", C.c_void_p), ("receiver_medium", C.c_void_p),
                ("receiver_qoffsets", C.c_void_p), ("receiver_quantities", C.c_void_p),
                ("record_every", C.c_int32), ("energy_every", C.c_int32)]


class _CArray(C.Structure):
    _fields_ = [("key", C.c_char_p), ("dtype", C.c_int32), ("n", C.c_int64), ("data", C.c_void_p)]


_DT = {0: np.float32, 1: np.float64, 2: np.int32, 3: np.uint8}


def setup_arrays(model: Model) -> Dict[str, np.ndarray]:
    """Runs the native setup; returns the flat problem layout (dt not set)."""
    d, keep = describe(model)
    L = cases_lib()
    out = C.c_void_p()
    if L.insem_case_build(C.byref(d), C.byref(out)) != 0:
        raise N.InsemError(N.ERR_INVALID, L.insem_case_last_error().decode())
    try:
        res = {}
        for i in range(L.insem_case_n_arrays(out)):
            a = _CArray.from_address(L.insem_case_array_at(out, i))
            dt = _DT[a.dtype]
            if a.n:
                buf = (C.c_char * (a.n * np.dtype(dt).itemsize)).from_address(a.data)
                res[a.key.decode()] = np.frombuffer(buf, dtype=dt).copy()
            else:
                res[a.key.decode()] = np.zeros(0, dt)
    finally:
        L.insem_case_free(out)
    for ri, r in enumerate(model.receivers):
        res[f"problem.receivers.{ri}.name"] = np.asarray(r.name)
        res[f"problem.receivers.{ri}.quantities"] = np.asarray(r.quantities, dtype="U32")
    for si in range(len(model.sources)):
        stf = model.sources[si].stf
        res[f"problem.sources.{si}.stf.samples"] = stf[4] if stf[0] == "samples" else np.zeros(0)
        res[f"problem.sources.{si}.stf.sample_dt"] = np.asarray(stf[5] if stf[0] == "samples" else 0.0)
    return res


def describe(model: Model):
    """The model as an ``insem_case_desc`` struct, plus the arrays it points into."""
    keep = []

    def arr(a, dtype):
        a = np.ascontiguousarray(np.asarray(a, dtype))
        keep.append(a)
        return a.ctypes.data if a.size else None

    m = model.mesh
    d = _Desc()
    d.quad9, d.axisymmetric = int(m.quad9), int(m.axisymmetric)
    d.n_nodes, d.nodes = m.nodes.shape[0], arr(m.nodes, np.float64)
    d.n_cells, d.cells, d.cell_region = m.cells.shape[0], arr(m.cells, np.int32), arr(m.region, np.int32)
    d.n_boundary, d.boundary = m.boundary.shape[0], arr(m.boundary, np.int32)
    d.order, d.uniform_level, d.f_max = model.order, model.uniform_level, model.f_max
    d.points_per_wavelength, d.max_level = model.points_per_wavelength, model.max_level
    d.n_regions, d.regions = len(model.regions), arr(np.asarray(model.regions, float).reshape(-1, 5), np.float64)
    d.azimuthal_order = model.azimuthal_order
    mats = sorted(model.materials.items())
    d.n_materials = len(mats)
    d.material_region = arr([r for r, _ in mats], np.int32)
    d.material_medium = arr([MEDIUM[x.medium] for _, x in mats], np.int32)
    d.material_vp = arr([x.vp for _, x in mats], np.float64)
    d.material_vs = arr([x.vs for _, x in mats], np.float64)
    d.material_rho = arr([x.rho for _, x in mats], np.float64)
    bcs = sorted(model.boundaries.items())
    d.n_bc, d.bc_tag, d.bc_type = len(bcs), arr([t for t, _ in bcs], np.int32), arr([BC[b] for _, b in bcs], np.int32)
    src = model.sources
    d.n_sources = len(src)
    d.source_kind = arr([SOURCE_KIND[s.kind] for s in src], np.int32)
    d.source_position = arr([[s.x, s.z] for s in src], np.float64)
    d.source_components = arr([list(s.components) for s in src], np.float64)
    d.stf_kind = arr([STF_KIND[s.stf[0]] for s in src], np.int32)
    d.stf_params = arr([[s.stf[1], s.stf[2] if s.stf[2] >= 0 or s.stf[0] == "samples" else 1.2 / s.stf[1], s.stf[3]]
                        for s in src], np.float64)
    rec = model.receivers
    d.n_receivers = len(rec)
    d.receiver_position = arr([[r.x, r.z] for r in rec], np.float64)
    d.receiver_medium = arr([MEDIUM.get(r.medium, -1) for r in rec], np.int32)
    qoff = np.cumsum([0] + [len(r.quantities) for r in rec])
    d.receiver_qoffsets = arr(qoff, np.int32)
    d.receiver_quantities = arr([N.QUANTITIES[q] for r in rec for q in r.quantities], np.int32)
    d.record_every, d.energy_every = model.record_every, model.energy_every
    return d, keep


def build(model: Model, device: int = 0, stable_dt: Optional[float] = None) -> ProblemData:
    """Native setup, then dt = safety x the device power-iteration estimate (or model.dt)."""
    return build_from_arrays(model, setup_arrays(model), device, stable_dt)


def build_from_arrays(model: Model, arrays: Dict[str, np.ndarray], device: int = 0,
                      stable_dt: Optional[float] = None) -> ProblemData:
    """``build`` on the output of ``setup_arrays`` (which may run in worker threads)."""
    from .solver import estimate_stable_dt

    arrays = dict(arrays)
    arrays["problem.dt"] = np.asarray(1.0)
    arrays["problem.n_steps"] = np.asarray(0)
    arrays["problem.stable_dt"] = np.asarray(0.0)
    prob = ProblemData.from_npz(arrays)
    sdt = stable_dt if stable_dt is not None else estimate_stable_dt(prob, device)
    prob.stable_dt = sdt
    if model.dt > 0.0:
        if model.dt > sdt:
            raise N.InsemError(N.ERR_INVALID, f"time step {model.dt} s exceeds the stability limit {sdt} s")
        prob.dt = model.dt
    else:
        prob.dt = model.safety * sdt
    if model.n_steps > 0:
        prob.n_steps = model.n_steps
    elif model.duration > 0.0:
        prob.n_steps = int(np.ceil(model.duration / prob.dt - 1e-9))
    return prob


def build_solver_from_arrays(model: Model, arrays: Dict[str, np.ndarray], device: int = 0, **solver_kwargs):
    """``build_from_arrays`` and ``Solver`` in one device construction: the
    solver estimates the stable time step from the arrays it uploads and
    applies the model's time settings (solver.cpp:131-144).  Same problem and
    solver as the two-step route, with one upload instead of two.  Returns
    (problem, solver)."""
    from .solver import Solver

    arrays = dict(arrays)
    arrays["problem.dt"] = np.asarray(1.0)
    arrays["problem.n_steps"] = np.asarray(0)
    arrays["problem.stable_dt"] = np.asarray(0.0)
    prob = ProblemData.from_npz(arrays)
    s = Solver(prob, device=device, time=(model.dt if model.dt > 0.0 else 0.0, model.safety,
                                          max(int(model.n_steps), 0), max(float(model.duration), 0.0)),
               **solver_kwargs)
    return prob, s


# --------------------------------------------------------------- workloads
MUD = Material.acoustic(1500.0, 1000.0)
STEEL = Material.elastic(5900.0, 3200.0, 7850.0)
CEMENT = Material.elastic(3000.0, 1600.0, 1900.0)
FAST = Material.elastic(4000.0, 2300.0, 2400.0)


def config1() -> Model:
    m = rectangle((-4.0, 4.0), (-4.0, 4.0), nx=32, nz=32)
    return Model(m, order=4, materials={0: Material.acoustic(1500.0, 1000.0)},
                 boundaries={t: "absorbing" for t in (BOTTOM, RIGHT, TOP, LEFT)},
                 sources=[Source("monopole", 0.0, 0.0, stf=ricker(400.0))],
                 receivers=[Receiver("h1", 1.5, 0.0, ["pressure"])], duration=4e-3)


def config2(z=(-1.5, 4.5), formation_radius=4.0) -> Model:
    b = borehole(z, [("mud", 0.1), ("casing", 0.11), ("cement", 0.14)], formation_radius=formation_radius, dz=0.08)
    mats = {b.regions["mud"]: MUD, b.regions["casing"]: STEEL, b.regions["cement"]: CEMENT,
            b.regions["formation"]: FAST}
    recs = [Receiver(f"r{i}", 0.05, 2.0 + 0.15 * i, ["pressure"]) for i in range(13)]
    return Model(b.mesh, order=4, f_max=7500.0, materials=mats,
                 boundaries={b.boundaries[n]: "absorbing" for n in ("bottom", "outer", "top")},
                 sources=[Source("monopole", 0.0, 0.0, stf=ricker(8000.0))], receivers=recs, duration=5e-3)


def config3_spec(nx: int = 1024, seed: int = 3, n_receivers: int = 512) -> dict:
    """The seeded layer stack of the large coupled model as plain data:
    interfaces (bottom to top; constants or vectorised z(x)), rows per layer,
    region ids, (vp, vs, rho) per elastic region and the receiver x positions."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(2.0, 6.0, 7)
    lam = rng.uniform(80.0, 200.0, 7)
    vp = rng.uniform(2000.0, 5500.0, 8)
    vs = vp * rng.uniform(0.45, 0.6, 8)
    rho = rng.uniform(2000.0, 2700.0, 8)
    zk = -340.0 + 340.0 * np.arange(1, 8) / 8.0
    interfaces: list = [-340.0]
    for k in range(7):
        interfaces.append(lambda x, z0=zk[k], a=amp[k], l=lam[k]: z0 + a * np.sin(2.0 * np.pi * x / l))
    interfaces += [0.0, 60.0]
    rows_water = round(154 * nx / 1024)
    rows_el = nx - rows_water
    counts = [rows_el // 8 + (1 if k < rows_el % 8 else 0) for k in range(8)] + [rows_water]
    return dict(interfaces=interfaces, counts=counts, regions=list(range(1, 9)) + [0],
                elastic={k + 1: (float(vp[k]), float(vs[k]), float(rho[k])) for k in range(8)},
                receivers_x=[float(x) for x in np.linspace(1.0, 399.0, n_receivers)])


def config3(nx: int = 1024, n_steps: int = 2000, seed: int = 3, n_receivers: int = 512) -> Model:
    """Water (60 m, 154/1024 of the rows) over 8 elastic layers with sinusoidal
    interfaces (amplitude U(2, 6) m, wavelength U(80, 200) m), 400 m wide, order 5,
    Quad9 cells; force source at (200, -20) Ricker 30 Hz; velocity receivers on
    the seafloor; Stacey on sides and bottom, free surface on top.  nx = 1024 is
    the benchmark size; rows scale with nx."""
    spec = config3_spec(nx, seed, n_receivers)
    m = layered((0.0, 400.0), spec["interfaces"], spec["counts"], spec["regions"], nx=nx, quadratic=True)
    mats = {0: Material.acoustic(1500.0, 1000.0)}
    for region, (vp, vs, rho) in spec["elastic"].items():
        mats[region] = Material.elastic(vp, vs, rho)
    recs = [Receiver(f"sf{i}", x, -0.5, ["velocity"], "elastic") for i, x in enumerate(spec["receivers_x"])]
    return Model(m, order=5, materials=mats,
                 boundaries={BOTTOM: "absorbing", LEFT: "absorbing", RIGHT: "absorbing", TOP: "free"},
                 sources=[Source("force", 200.0, -20.0, (0.0, 1.0, 0.0), ricker(30.0))], receivers=recs,
                 n_steps=n_steps)


# ------------------------------------------------------------ config 4
C4_RECEIVERS_Z = (2.0, 0.15, 13)  # first z, spacing, count (r = 0.05 m, in the mud)
C4_ELEMENTS = (5000, 80000)


def config4_params(n_models: int = 256, seed: int = 4) -> List[dict]:
    """Seeded draws of the batched borehole workload: hole radius U(0.08, 0.15) m;
    azimuthal order 0 (monopole, Ricker 8 kHz) or 1 (dipole, Ricker 3 kHz), half
    each; 1-6 horizontal beds with vp U(2000, 5500), vs/vp U(0.4, 0.6), rho
    U(2000, 2700) (slow formations, vs < 1500, included); a 0.01 m steel casing
    and 0.03 m cement in 30 % of the models; GLL order 4-6; a target size of
    5k-80k elements after AMR (log-uniform); 13 pressure receivers; 5 ms."""
    rng = np.random.default_rng(seed)
    orders_m = rng.permutation(np.arange(n_models) % 2)
    out = []
    for k in range(n_models):
        nb = int(rng.integers(1, 7))
        vp = rng.uniform(2000.0, 5500.0, nb)
        vs = vp * rng.uniform(0.4, 0.6, nb)
        rho = rng.uniform(2000.0, 2700.0, nb)
        out.append(dict(
            index=k,
            m=int(orders_m[k]),
            hole=float(rng.uniform(0.08, 0.15)),
            casing=bool(rng.random() < 0.3),
            order=int(rng.integers(4, 7)),
            beds=[(float(a), float(b), float(c)) for a, b, c in zip(vp, vs, rho)],
            bed_fracs=sorted(float(f) for f in rng.uniform(0.1, 0.9, nb - 1)),
            target=float(np.exp(rng.uniform(np.log(C4_ELEMENTS[0]), np.log(C4_ELEMENTS[1])))),
        ))
    return out


def config4_model(p: dict, zlen: float = 6.0, radius: float = 4.0, duration: float = 5e-3) -> Model:
    """One batched borehole model: z from -1.5 m over `zlen`, formation out to `radius`."""
    hole = p["hole"]
    ann = [("mud", hole)] + ([("casing", hole + 0.01), ("cement", hole + 0.04)] if p["casing"] else [])
    z0 = -1.5
    beds = [(z0, "bed0")] + [(z0 + zlen * f, f"bed{i + 1}") for i, f in enumerate(p["bed_fracs"])]
    b = borehole((z0, z0 + zlen), ann, formation_radius=radius, beds=beds, dz=0.08)
    mats = {b.regions["mud"]: MUD}
    if p["casing"]:
        mats[b.regions["casing"]] = STEEL
        mats[b.regions["cement"]] = CEMENT
    for i, (vp, vs, rho) in enumerate(p["beds"]):
        mats[b.regions[f"bed{i}"]] = Material.elastic(vp, vs, rho)
    if p["m"] == 0:
        f0 = 8000.0
        src = Source("monopole", 0.0, 0.0, stf=ricker(f0))
    else:
        f0 = 3000.0
        src = Source("dipole", 0.0, 0.0, (1.0, 0.0, 0.0), ricker(f0))
    z_first, dz_rec, n_rec = C4_RECEIVERS_Z
    recs = [Receiver(f"r{i}", 0.05, z_first + dz_rec * i, ["pressure"]) for i in range(n_rec)]
    return Model(b.mesh, order=p["order"], f_max=0.9375 * f0, azimuthal_order=p["m"], materials=mats,
                 boundaries={b.boundaries[n]: "absorbing" for n in ("bottom", "outer", "top")},
                 sources=[src], receivers=recs, duration=duration)


def n_elements(arrays: Dict[str, np.ndarray]) -> int:
    return int(sum(v.size for k, v in arrays.items() if k.endswith(".elements")))


def config4_calibrated(p: dict, duration: float = 5e-3, geometry: Optional[Tuple[float, float]] = None):
    """(model, setup arrays, elements, (zlen, radius)).  Without `geometry`, the z
    extent and formation radius are scaled (at most three setups) so the mesh
    after AMR lands near the model's target size, inside 5k-80k elements."""
    if geometry is not None:
        model = config4_model(p, geometry[0], geometry[1], duration)
        arrays = setup_arrays(model)
        return model, arrays, n_elements(arrays), geometry
    lo, hi = C4_ELEMENTS
    zlen, radius = 6.0, 4.0
    model = config4_model(p, zlen, radius, duration)
    arrays = setup_arrays(model)
    ne = n_elements(arrays)
    for it in range(3):
        if lo <= ne <= hi and (it == 2 or abs(np.log(ne / p["target"])) < 0.35):
            break
        s = p["target"] / ne
        if s >= 1.0:
            g = s ** 0.5
            zlen, radius = min(zlen * g, 60.0), min(radius * g, 30.0)
        else:
            radius = max(radius * s, 0.6 + p["hole"])
        model = config4_model(p, zlen, radius, duration)
        arrays = setup_arrays(model)
        ne = n_elements(arrays)
    return model, arrays, ne, (zlen, radius)


C4_GEOMETRY_FILE = "config4_geometry.json"


def config4_geometry_table(n_models: int = 256, seed: int = 4) -> Optional[List[Tuple[float, float]]]:
    """The calibrated (zlen, radius) of every model, from the table shipped with
    the package (written by ``write_config4_geometry``), or None."""
    import json
    from pathlib import Path

    f = Path(__file__).resolve().parent / "data" / C4_GEOMETRY_FILE
    if not f.exists():
        return None
    t = json.loads(f.read_text())
    if t.get("seed") != seed or len(t.get("geometry", [])) < n_models:
        return None
    return [tuple(g) for g in t["geometry"][:n_models]]


def write_config4_geometry(n_models: int = 256, seed: int = 4) -> None:
    """Calibrates every model of the workload and writes the geometry table."""
    import json
    from pathlib import Path

    rows, counts = [], []
    for p, _, _, ne, geo in config4(n_models, seed, use_table=False):
        rows.append([round(geo[0], 6), round(geo[1], 6)])
        counts.append(ne)
    f = Path(__file__).resolve().parent / "data" / C4_GEOMETRY_FILE
    f.parent.mkdir(exist_ok=True)
    f.write_text(json.dumps({"seed": seed, "n_models": n_models, "geometry": rows, "elements": counts}) + "\n")


def config4(n_models: int = 256, seed: int = 4, workers: Optional[int] = None, duration: float = 5e-3,
            use_table: bool = True):
    """Yields (params, model, setup arrays, elements, (zlen, radius)) of the
    batched borehole workload in order; the native setups run in a thread pool."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    params = config4_params(n_models, seed)
    table = config4_geometry_table(n_models, seed) if use_table else None
    geos = table if table is not None else [None] * n_models
    with ThreadPoolExecutor(max_workers=workers or max(1, min(32, os.cpu_count() or 1))) as ex:
        results = ex.map(lambda qg: config4_calibrated(qg[0], duration, qg[1]), zip(params, geos))
        for p, (model, arrays, ne, geo) in zip(params, results):
            yield p, model, arrays, ne, geo
