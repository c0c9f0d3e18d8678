"""Host-side description of one solve: every array the per-step path reads.

The fields mirror what the reference's ``solver::Solver(Problem)`` constructor
builds (cpp/src/solver/solver.cpp:91-568): per domain the DofMap arrays
(dof_map.hpp:84-91), element blocks (element_block.hpp:31-46), lumped mass,
Stacey, Dirichlet and axis lists; the fluid-solid coupling; sources expanded
onto global points; receiver interpolation weights; dt and the step counts.
``to_c`` packs it into the ``insem_cuda_problem`` struct of the C ABI.

A problem is stored as flat ``.npz`` keys (``problem.domains.0.l2g`` ...), the
same layout the golden fixtures use.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import native as N

STF_KINDS = {"ricker": 0, "gaussian": 1, "gaussian_derivative": 2, "samples": 3}


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel())


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


@dataclass
class BlockData:
    kind: int
    azimuthal_order: int
    elements: np.ndarray
    metric: np.ndarray
    coef0: np.ndarray
    coef1: np.ndarray
    wr: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    hoop: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    r: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    axial: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint8))

    @property
    def n_elements(self) -> int:
        return int(self.elements.size)


@dataclass
class DomainData:
    medium: int
    ncomp: int
    azimuthal_order: int
    n_global: int
    n_elements: int
    l2g: np.ndarray
    row_offsets: np.ndarray
    row_dofs: np.ndarray
    row_weights: np.ndarray
    t_offsets: np.ndarray
    t_slots: np.ndarray
    t_weights: np.ndarray
    mass: np.ndarray
    inv_mass: np.ndarray
    absorbing_points: np.ndarray
    absorbing_coef: np.ndarray
    dirichlet_points: np.ndarray
    axis_points: np.ndarray
    axis_components: np.ndarray
    blocks: List[BlockData]

    @property
    def n_rows(self) -> int:
        return max(int(self.row_offsets.size) - 1, 0)


@dataclass
class SourceData:
    domain: int
    points: np.ndarray
    coef: np.ndarray  # [ncomp][n_points]
    stf_kind: int
    f0: float
    t0: float
    amplitude: float
    samples: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sample_dt: float = 0.0


@dataclass
class ReceiverData:
    name: str
    domain: int
    points: np.ndarray
    value: np.ndarray
    d_dx: np.ndarray
    d_dz: np.ndarray
    rho: float
    quantities: List[str]


@dataclass
class ProblemData:
    ngll: int
    D: np.ndarray
    Dj: np.ndarray
    w2: np.ndarray
    domains: List[DomainData]
    coupling: Dict[str, np.ndarray]
    sources: List[SourceData]
    receivers: List[ReceiverData]
    dt: float
    n_steps: int
    record_every: int = 1
    energy_every: int = 0
    axisym: bool = False
    azimuthal_order: int = 0
    stable_dt: float = 0.0

    # ------------------------------------------------------------ queries
    @property
    def media(self) -> List[str]:
        return ["acoustic" if d.medium == N.ACOUSTIC else "elastic" for d in self.domains]

    def domain_index(self, medium: str) -> int:
        code = N.ACOUSTIC if medium == "acoustic" else N.ELASTIC
        for i, d in enumerate(self.domains):
            if d.medium == code:
                return i
        return -1

    def n_global_total(self) -> int:
        """Unique global points summed over domains (the GLL-point count of the metric)."""
        return int(sum(d.n_global for d in self.domains))

    def n_elements_total(self) -> int:
        return int(sum(d.n_elements for d in self.domains))

    def trace_list(self) -> List[tuple]:
        """(receiver, quantity) of every trace, in the reference's order."""
        return [(r.name, q) for r in self.receivers for q in r.quantities]

    def algorithmic_bytes_per_step(self) -> int:
        """Minimum HBM bytes of one step (fp32):
        sum_domains n_g (16 ncomp + 4) + sum_elements [4 npe + metric(kind) + coef],
        metric Rect 12, Affine 20, Curved 20 npe, Axisym 28 npe (xi_r, xi_z,
        eta_r, eta_z, wr, hoop, r: the axisymmetric fluxes use the Jacobian only
        through wr); coef elastic 8 npe, acoustic 4 npe."""
        npe = self.ngll * self.ngll
        total = 0
        for d in self.domains:
            total += d.n_global * (16 * d.ncomp + 4)
            coef = (8 if d.medium == N.ELASTIC else 4) * npe
            for b in d.blocks:
                metric = {N.RECT: 12, N.AFFINE: 20, N.CURVED: 20 * npe, N.AXISYM: 28 * npe}[b.kind]
                total += b.n_elements * (4 * npe + metric + coef)
        return int(total)

    def algorithmic_bytes_split(self, tile_points) -> tuple:
        """(bytes of the tile kernels, bytes of the halo kernels) of one step: the
        element terms and the points finished in their tile, against the points
        finished by the halo kernel; tile_points[d] per domain."""
        npe = self.ngll * self.ngll
        tile = halo = 0
        for d, nt in zip(self.domains, tile_points):
            per_point = 16 * d.ncomp + 4
            tile += nt * per_point
            halo += (d.n_global - nt) * per_point
            coef = (8 if d.medium == N.ELASTIC else 4) * npe
            for b in d.blocks:
                metric = {N.RECT: 12, N.AFFINE: 20, N.CURVED: 20 * npe, N.AXISYM: 28 * npe}[b.kind]
                tile += b.n_elements * (4 * npe + metric + coef)
        return int(tile), int(halo)

    # ------------------------------------------------------------- storage
    @staticmethod
    def from_npz(z, prefix: str = "problem.") -> "ProblemData":
        """Reads the flat key layout of the golden fixtures."""
        def g(k):
            return z[prefix + k]

        def s(k):
            return g(k).item()

        nd = int(s("domains.count"))
        domains = []
        for di in range(nd):
            p = f"domains.{di}."
            nb = int(s(p + "blocks.count"))
            blocks = []
            for bi in range(nb):
                q = p + f"blocks.{bi}."
                blocks.append(BlockData(int(s(q + "kind")), int(s(q + "azimuthal_order")), _i32(g(q + "elements")),
                                        _f32(g(q + "metric")), _f32(g(q + "coef0")), _f32(g(q + "coef1")),
                                        _f32(g(q + "wr")), _f32(g(q + "hoop")), _f32(g(q + "r")),
                                        np.ascontiguousarray(g(q + "axial").astype(np.uint8))))
            domains.append(DomainData(
                int(s(p + "medium")), int(s(p + "ncomp")), int(s(p + "azimuthal_order")), int(s(p + "n_global")),
                int(s(p + "n_elements")), _i32(g(p + "l2g")), _i32(g(p + "row_offsets")), _i32(g(p + "row_dofs")),
                _f64(g(p + "row_weights")), _i32(g(p + "t_offsets")), _i32(g(p + "t_slots")),
                _f64(g(p + "t_weights")), _f32(g(p + "mass")), _f32(g(p + "inv_mass")),
                _i32(g(p + "absorbing_points")), _f32(g(p + "absorbing_coef")), _i32(g(p + "dirichlet_points")),
                _i32(g(p + "axis_points")), _i32(g(p + "axis_components")), blocks))
        sources = []
        for si in range(int(s("sources.count"))):
            p = f"sources.{si}."
            sources.append(SourceData(int(s(p + "domain")), _i32(g(p + "points")), _f32(g(p + "coef")),
                                      int(s(p + "stf.kind")), float(s(p + "stf.f0")), float(s(p + "stf.t0")),
                                      float(s(p + "stf.amplitude")), _f64(g(p + "stf.samples")),
                                      float(s(p + "stf.sample_dt"))))
        receivers = []
        for ri in range(int(s("receivers.count"))):
            p = f"receivers.{ri}."
            receivers.append(ReceiverData(str(s(p + "name")), int(s(p + "domain")), _i32(g(p + "points")),
                                          _f32(g(p + "value")), _f32(g(p + "d_dx")), _f32(g(p + "d_dz")),
                                          float(s(p + "rho")), [str(q) for q in g(p + "quantities")]))
        coupling = {k: g("coupling." + k) for k in ("fluid_points", "solid_points", "cx", "cz")}
        coupling = {k: (_i32(v) if "points" in k else _f32(v)) for k, v in coupling.items()}
        return ProblemData(int(s("basis.ngll")), _f32(g("basis.D")), _f32(g("basis.Dj")), _f32(g("basis.w2")),
                           domains, coupling, sources, receivers, float(s("dt")), int(s("n_steps")),
                           int(s("record_every")), int(s("energy_every")), bool(s("axisym")),
                           int(s("azimuthal_order")), float(s("stable_dt")))

    # ------------------------------------------------------------ C struct
    def to_c(self) -> "PackedProblem":
        return PackedProblem(self)


class PackedProblem:
    """The problem as an ``insem_cuda_problem`` struct; keeps the arrays alive."""

    def __init__(self, p: ProblemData):
        self._keep: list = []
        keep = self._keep

        def ptr(a, ctype):
            if a is None or np.asarray(a).size == 0:
                return C.cast(None, C.POINTER(ctype))
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(ctype))

        c = N.Problem()
        c.basis = N.Basis(p.ngll, ptr(_f32(p.D), C.c_float), ptr(_f32(p.Dj), C.c_float), ptr(_f32(p.w2), C.c_float))
        doms = (N.Domain * len(p.domains))()
        for i, d in enumerate(p.domains):
            blocks = (N.Block * max(len(d.blocks), 1))()
            for j, b in enumerate(d.blocks):
                blocks[j] = N.Block(b.kind, b.azimuthal_order, b.n_elements, ptr(_i32(b.elements), C.c_int32),
                                    ptr(_f32(b.metric), C.c_float), ptr(_f32(b.coef0), C.c_float),
                                    ptr(_f32(b.coef1), C.c_float), ptr(_f32(b.wr), C.c_float),
                                    ptr(_f32(b.hoop), C.c_float), ptr(_f32(b.r), C.c_float),
                                    ptr(np.ascontiguousarray(b.axial, np.uint8), C.c_uint8))
            keep.append(blocks)
            weighted = d.n_rows > 0 and d.t_weights.size > 0
            dm = N.DofMap(p.ngll, d.n_elements, d.n_global, ptr(_i32(d.l2g), C.c_int32), d.n_rows,
                          ptr(_i32(d.row_offsets), C.c_int32), ptr(_i32(d.row_dofs), C.c_int32),
                          ptr(_f64(d.row_weights), C.c_double), ptr(_i32(d.t_offsets), C.c_int32),
                          ptr(_i32(d.t_slots), C.c_int32),
                          ptr(_f64(d.t_weights), C.c_double) if weighted else C.cast(None, N.f64p))
            doms[i] = N.Domain(d.medium, d.ncomp, d.azimuthal_order, dm, len(d.blocks), blocks,
                               ptr(_f32(d.mass), C.c_float), ptr(_f32(d.inv_mass), C.c_float),
                               int(d.absorbing_points.size), ptr(_i32(d.absorbing_points), C.c_int32),
                               ptr(_f32(d.absorbing_coef), C.c_float), int(d.dirichlet_points.size),
                               ptr(_i32(d.dirichlet_points), C.c_int32), int(d.axis_points.size),
                               ptr(_i32(d.axis_points), C.c_int32), int(d.axis_components.size),
                               ptr(_i32(d.axis_components), C.c_int32))
        keep.append(doms)
        c.n_domains = len(p.domains)
        c.domains = doms
        cp = p.coupling
        c.coupling = N.Coupling(int(cp["fluid_points"].size), ptr(_i32(cp["fluid_points"]), C.c_int32),
                                ptr(_i32(cp["solid_points"]), C.c_int32), ptr(_f32(cp["cx"]), C.c_float),
                                ptr(_f32(cp["cz"]), C.c_float))
        srcs = (N.Source * max(len(p.sources), 1))()
        for i, s in enumerate(p.sources):
            stf = N.Stf(s.stf_kind, s.f0, s.t0, s.amplitude, int(s.samples.size), ptr(_f64(s.samples), C.c_double),
                        s.sample_dt)
            srcs[i] = N.Source(s.domain, int(s.points.size), ptr(_i32(s.points), C.c_int32),
                               ptr(_f32(s.coef), C.c_float), stf)
        keep.append(srcs)
        c.n_sources = len(p.sources)
        c.sources = srcs
        recs = (N.Receiver * max(len(p.receivers), 1))()
        for i, r in enumerate(p.receivers):
            q = _i32([N.QUANTITIES[x] for x in r.quantities])
            recs[i] = N.Receiver(r.domain, int(r.points.size), ptr(_i32(r.points), C.c_int32),
                                 ptr(_f32(r.value), C.c_float), ptr(_f32(r.d_dx), C.c_float),
                                 ptr(_f32(r.d_dz), C.c_float), r.rho, int(q.size), ptr(q, C.c_int32))
        keep.append(recs)
        c.n_receivers = len(p.receivers)
        c.receivers = recs
        c.dt = p.dt
        c.n_steps = p.n_steps
        c.record_every = p.record_every
        c.energy_every = p.energy_every
        self.struct = c

    def ref(self):
        return C.byref(self.struct)
