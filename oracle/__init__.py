"""The oracle: a CPU restatement of insem's per-time-step path (insem_oracle.c).

TEST INFRASTRUCTURE ONLY -- the checker of the CUDA backend, never part of
the product path.  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use it.  It is pinned against the reference's own outputs
(tests/golden, generated from the reference build in oracle/ref) by
tests/test_oracle_golden.py.

``OracleSolver`` mirrors the device solver's Python API; ``block_forces``,
``gather``, ``assemble`` mirror the kernel seams.  Inputs are the packed
problem structs of include/insem_cuda.h (built by the package's problem.py).
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
        L = C.CDLL(str(LIB))
        vp = C.c_void_p
        f32p = C.POINTER(C.c_float)
        f64p = C.POINTER(C.c_double)
        L.oracle_block_forces.argtypes = [vp, vp, C.c_int32, f32p, f32p]
        L.oracle_block_forces.restype = C.c_int
        L.oracle_gather.argtypes = [vp, C.c_int32, f32p, f32p]
        L.oracle_assemble.argtypes = [vp, C.c_int32, f32p, f32p]
        L.oracle_solver_create.argtypes = [vp]
        L.oracle_solver_create.restype = vp
        L.oracle_solver_destroy.argtypes = [vp]
        L.oracle_solver_set_state.argtypes = [vp, C.c_int32, f64p, f64p]
        L.oracle_solver_set_state.restype = C.c_int
        L.oracle_solver_advance.argtypes = [vp, C.c_int32]
        for name in ("oracle_solver_step", "oracle_solver_n_cols", "oracle_solver_n_samples", "oracle_solver_n_energy"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = C.c_int32
        L.oracle_solver_samples.argtypes = [vp, f64p]
        L.oracle_solver_energy.argtypes = [vp, f64p]
        L.oracle_solver_state.argtypes = [vp, C.c_int32, f32p, f32p, f32p]
        L.oracle_internal_forces.argtypes = [vp, C.c_int32, f32p, f32p]
        _lib = L
    return _lib


def _f32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class OracleSolver:
    """CPU time loop over a ProblemData (same API subset as the device Solver)."""

    def __init__(self, problem):
        self.problem = problem
        self._packed = problem.to_c()
        self._h = C.c_void_p(lib().oracle_solver_create(C.addressof(self._packed.struct)))
        self._traces = problem.trace_list()
        ncomp = {}
        for r in problem.receivers:
            d = problem.domains[r.domain]
            for q in r.quantities:
                ncomp[(r.name, q)] = 2 if q == "particle_velocity" else d.ncomp
        self._ncomp = ncomp

    def __del__(self):
        if getattr(self, "_h", None):
            lib().oracle_solver_destroy(self._h)
            self._h = None

    def set_state(self, medium: str, u, v) -> None:
        code = 0 if medium == "acoustic" else 1
        u = np.ascontiguousarray(np.asarray(u, np.float64).ravel())
        v = np.ascontiguousarray(np.asarray(v, np.float64).ravel())
        rc = lib().oracle_solver_set_state(self._h, code, u.ctypes.data_as(C.POINTER(C.c_double)),
                                           v.ctypes.data_as(C.POINTER(C.c_double)))
        if rc:
            raise RuntimeError(f"oracle set_state failed ({rc})")

    def advance(self, n: int) -> None:
        lib().oracle_solver_advance(self._h, int(n))

    def run(self) -> None:
        self.advance(self.problem.n_steps - self.step)

    @property
    def step(self) -> int:
        return int(lib().oracle_solver_step(self._h))

    def _samples(self) -> np.ndarray:
        ns, nc = lib().oracle_solver_n_samples(self._h), lib().oracle_solver_n_cols(self._h)
        out = np.empty((ns, nc))
        lib().oracle_solver_samples(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def trace(self, receiver: str, quantity: str) -> np.ndarray:
        s = self._samples()
        col = 0
        for key in self._traces:
            nc = self._ncomp[key]
            if key == (receiver, quantity):
                return np.ascontiguousarray(s[:, col:col + nc])
            col += nc
        raise KeyError((receiver, quantity))

    @property
    def energy(self) -> np.ndarray:
        n = lib().oracle_solver_n_energy(self._h)
        out = np.empty((n, 3))
        lib().oracle_solver_energy(self._h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def state(self, domain: int):
        d = self.problem.domains[domain]
        arrs = [np.empty(d.ncomp * d.n_global, np.float32) for _ in range(3)]
        lib().oracle_solver_state(self._h, domain, *[_f32p(a) for a in arrs])
        return tuple(a.astype(np.float64).reshape(d.ncomp, d.n_global) for a in arrs)

    def internal_forces(self, domain: int, u) -> np.ndarray:
        d = self.problem.domains[domain]
        u = np.ascontiguousarray(np.asarray(u, np.float32).ravel())
        f = np.empty(d.ncomp * d.n_global, np.float32)
        lib().oracle_internal_forces(self._h, domain, _f32p(u), _f32p(f))
        return f


def block_forces(problem, domain: int, block: int, u_local) -> np.ndarray:
    """f_local of one block (physics::*_internal_forces) on the CPU."""
    packed = problem.to_c()
    dom = packed.struct.domains[domain]
    d = problem.domains[domain]
    f = np.zeros(d.ncomp * d.l2g.size, np.float32)
    u = np.ascontiguousarray(np.asarray(u_local, np.float32).ravel())
    rc = lib().oracle_block_forces(C.addressof(packed.struct.basis), C.addressof(dom.blocks[block]), d.medium,
                                   _f32p(u), _f32p(f))
    if rc:
        raise RuntimeError(f"oracle block_forces failed ({rc})")
    return f


def gather(problem, domain: int, g) -> np.ndarray:
    packed = problem.to_c()
    d = problem.domains[domain]
    g = np.ascontiguousarray(np.asarray(g, np.float32).ravel())
    out = np.empty(d.ncomp * d.l2g.size, np.float32)
    lib().oracle_gather(C.addressof(packed.struct.domains[domain].dofs), d.ncomp, _f32p(g), _f32p(out))
    return out


def assemble(problem, domain: int, local) -> np.ndarray:
    packed = problem.to_c()
    d = problem.domains[domain]
    local = np.ascontiguousarray(np.asarray(local, np.float32).ravel())
    out = np.empty(d.ncomp * d.n_global, np.float32)
    lib().oracle_assemble(C.addressof(packed.struct.domains[domain].dofs), d.ncomp, _f32p(local), _f32p(out))
    return out
