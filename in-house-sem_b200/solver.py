"""Python face of the device solver, shaped like the reference's ``insem.Solver``
binding (python/src/bindings.cpp:330-398): ``dt``, ``n_steps``, ``step``,
``time``, ``advance``, ``run``, ``media``, ``state``, ``set_state``,
``trace``, ``times``, ``energy``.  Every call goes through the C ABI.
"""

from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import native as N
from .problem import ProblemData


class Solver:
    def __init__(self, problem: ProblemData, device: int = 0, use_graphs: bool = True, path: int = 0,
                 tile_elements: int = 0, check_finite: bool = True, time: Optional[Tuple[float, float, int, float]] = None):
        """``time`` = (dt, safety, n_steps, duration), the reference's time
        settings: the solver then estimates the stable time step on the device
        and derives dt and n_steps as the reference Solver constructor does
        (solver.cpp:131-144); ``problem`` gets dt, n_steps and stable_dt."""
        self.problem = problem
        self._packed = problem.to_c()
        opts = N.Options(device, int(use_graphs), path, tile_elements, int(check_finite))
        h = C.c_void_p()
        if time is None:
            N.check(N.lib().insem_cuda_solver_create(self._packed.ref(), C.byref(opts), C.byref(h)))
        else:
            t = N.Time(float(time[0]), float(time[1]), int(time[2]), float(time[3]))
            N.check(N.lib().insem_cuda_solver_create_timed(self._packed.ref(), C.byref(t), C.byref(opts), C.byref(h)))
            problem.dt = float(N.lib().insem_cuda_solver_dt(h))
            problem.n_steps = int(N.lib().insem_cuda_solver_n_steps(h))
            problem.stable_dt = float(N.lib().insem_cuda_solver_stable_dt(h))
        self._h = h
        self._traces = problem.trace_list()

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().insem_cuda_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------- properties
    @property
    def dt(self) -> float:
        return float(N.lib().insem_cuda_solver_dt(self._h))

    @property
    def stable_dt(self) -> float:
        return float(self.problem.stable_dt)

    @property
    def n_steps(self) -> int:
        return int(N.lib().insem_cuda_solver_n_steps(self._h))

    @property
    def step(self) -> int:
        return int(N.lib().insem_cuda_solver_step(self._h))

    @property
    def failed(self) -> bool:
        """A finite check found NaN or Inf in this solve's fields."""
        return int(N.lib().insem_cuda_solver_status(self._h)) == N.ERR_NONFINITE

    @property
    def time(self) -> float:
        return self.step * self.dt

    @property
    def media(self):
        return self.problem.media

    @property
    def last_advance_ms(self) -> float:
        return float(N.lib().insem_cuda_solver_last_advance_ms(self._h))

    # ---------------------------------------------------------- stepping
    def advance(self, n_steps: int) -> None:
        N.check(N.lib().insem_cuda_solver_advance(self._h, int(n_steps)))

    def run(self) -> None:
        N.check(N.lib().insem_cuda_solver_run(self._h))

    def prepare_for_batch(self) -> None:
        """Runs the initial step and the predictor now (on this solver's
        stream), so that joining a batch later costs the batch nothing;
        afterwards only a batch steps this solver."""
        N.check(N.lib().insem_cuda_solver_prepare_for_batch(self._h))

    def advance_streamed(self, n_steps: int, amplitudes: np.ndarray, rows_out: np.ndarray) -> int:
        """n steps with per-step source amplitudes in ([n][n_sources] float32, host) and
        the recorded rows out ([>= n / record_every][n_columns] float64, host)."""
        assert amplitudes.dtype == np.float32 and amplitudes.flags.c_contiguous
        assert rows_out.dtype == np.float64 and rows_out.flags.c_contiguous
        n = C.c_int32()
        N.check(N.lib().insem_cuda_solver_advance_streamed(self._h, int(n_steps), amplitudes.ctypes.data_as(N.f32p),
                                                           rows_out.ctypes.data_as(N.f64p), C.byref(n)))
        return n.value

    @property
    def n_columns(self) -> int:
        return int(N.lib().insem_cuda_solver_n_columns(self._h))

    @property
    def kernels_per_step(self) -> int:
        return int(N.lib().insem_cuda_solver_kernels_per_step(self._h))

    def point_classes(self, domain: int) -> Tuple[int, int]:
        """(points finished in their tile, points finished by the halo kernel)."""
        nt, nh = C.c_int32(), C.c_int32()
        N.check(N.lib().insem_cuda_solver_point_classes(self._h, int(domain), C.byref(nt), C.byref(nh)))
        return nt.value, nh.value

    def algorithmic_bytes_split(self) -> Tuple[int, int]:
        """(tile-kernel bytes, halo-kernel bytes) of one step (the roofline's split)."""
        return self.problem.algorithmic_bytes_split(
            [self.point_classes(i)[0] for i in range(len(self.problem.domains))])

    # ------------------------------------------------------------- state
    def _domain(self, medium: str) -> int:
        di = self.problem.domain_index(medium)
        if di < 0:
            raise N.InsemError(N.ERR_INVALID, f"the model has no {medium} region")
        return di

    def state(self, medium: str) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        d = self.problem.domains[self._domain(medium)]
        shape = (d.ncomp, d.n_global)
        u, v, a = (np.empty(shape) for _ in range(3))
        N.check(N.lib().insem_cuda_solver_state(self._h, self._domain(medium), u.ctypes.data_as(N.f64p),
                                                v.ctypes.data_as(N.f64p), a.ctypes.data_as(N.f64p)))
        return u, v, a

    def set_state(self, medium: str, u, v) -> None:
        d = self.problem.domains[self._domain(medium)]
        u = np.ascontiguousarray(np.asarray(u, np.float64).reshape(-1))
        v = np.ascontiguousarray(np.asarray(v, np.float64).reshape(-1))
        n = d.ncomp * d.n_global
        if u.size != n or v.size != n:
            raise N.InsemError(N.ERR_INVALID, f"state arrays must have {d.ncomp} x {d.n_global} entries")
        code = N.ACOUSTIC if medium == "acoustic" else N.ELASTIC
        N.check(N.lib().insem_cuda_solver_set_state(self._h, code, u.ctypes.data_as(N.f64p),
                                                    v.ctypes.data_as(N.f64p)))

    # ------------------------------------------------------------ outputs
    @property
    def n_samples(self) -> int:
        return int(N.lib().insem_cuda_solver_n_samples(self._h))

    def trace_by_index(self, t: int) -> np.ndarray:
        nc = int(N.lib().insem_cuda_solver_trace_ncomp(self._h, t))
        out = np.empty((self.n_samples, nc))
        N.check(N.lib().insem_cuda_solver_trace(self._h, t, out.ctypes.data_as(N.f64p)))
        return out

    def trace(self, receiver: str, quantity: str) -> np.ndarray:
        for t, (r, q) in enumerate(self._traces):
            if r == receiver and q == quantity:
                return self.trace_by_index(t)
        raise N.InsemError(N.ERR_INVALID, f"no trace '{quantity}' for receiver '{receiver}'")

    def traces(self) -> list:
        return [self.trace_by_index(t) for t in range(len(self._traces))]

    @property
    def times(self) -> np.ndarray:
        out = np.empty(self.n_samples)
        N.check(N.lib().insem_cuda_solver_times(self._h, out.ctypes.data_as(N.f64p)))
        return out

    @property
    def energy(self) -> np.ndarray:
        n = C.c_int32()
        N.check(N.lib().insem_cuda_solver_energy(self._h, None, 0, C.byref(n)))
        out = np.empty((n.value, 3))
        if n.value:
            N.check(N.lib().insem_cuda_solver_energy(self._h, out.ctypes.data_as(N.f64p), n.value, C.byref(n)))
        return out

    # --------------------------------------------------------- snapshots
    def set_snapshots(self, every: int, quantities=("velocity", "pressure")) -> None:
        """Wavefield snapshots every `every` steps and at step 0 (the
        reference's TimeConfig snapshot_every / snapshot_quantities); before
        the first step."""
        q = np.ascontiguousarray([N.QUANTITIES[x] for x in quantities], np.int32)
        N.check(N.lib().insem_cuda_solver_set_snapshots(self._h, int(every), int(q.size), q.ctypes.data_as(N.i32p)))

    @property
    def snapshot_times(self) -> np.ndarray:
        out = np.empty(int(N.lib().insem_cuda_solver_n_snapshots(self._h)))
        N.check(N.lib().insem_cuda_solver_snapshot_times(self._h, out.ctypes.data_as(N.f64p)))
        return out

    def snapshot(self, medium: str, quantity: str) -> np.ndarray:
        """(n_snapshots, ncomp, n_points) snapshot data, as the reference's Solver.snapshot."""
        want = (N.ACOUSTIC if medium == "acoustic" else N.ELASTIC, N.QUANTITIES[quantity])
        for f in range(int(N.lib().insem_cuda_solver_n_snapshot_fields(self._h))):
            med, qu, nc, npts = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int64()
            N.check(N.lib().insem_cuda_solver_snapshot_field(self._h, f, C.byref(med), C.byref(qu), C.byref(nc),
                                                             C.byref(npts)))
            if (med.value, qu.value) != want:
                continue
            ns = int(N.lib().insem_cuda_solver_n_snapshots(self._h))
            out = np.empty((ns, nc.value, npts.value), np.float32)
            N.check(N.lib().insem_cuda_solver_snapshot(self._h, f, out.ctypes.data_as(N.f32p)))
            return out
        raise N.InsemError(N.ERR_INVALID, f"no {quantity} snapshots for the {medium} medium")

    def internal_forces(self, domain: int, u: np.ndarray) -> np.ndarray:
        d = self.problem.domains[domain]
        u = np.ascontiguousarray(np.asarray(u, np.float32).reshape(-1))
        f = np.empty(d.ncomp * d.n_global, np.float32)
        N.check(N.lib().insem_cuda_solver_internal_forces(self._h, domain, u.ctypes.data_as(N.f32p),
                                                          f.ctypes.data_as(N.f32p)))
        return f


def estimate_stable_dt(problem: ProblemData, device: int = 0) -> float:
    """2 / sqrt(lambda_max(M^-1 K)) by the reference's power iteration, on the device."""
    packed = problem.to_c()
    out = C.c_double()
    N.check(N.lib().insem_cuda_stable_dt(packed.ref(), device, C.byref(out)))
    return float(out.value)
