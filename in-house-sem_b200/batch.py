"""Batched solves: many independent problems advanced by shared launches.

Every batched step is one CUDA graph with a fixed number of launches,
whatever the number of problems:
- one tile kernel per tile class, one CTA per tile; the classes spread over
  ``tile_streams`` streams (default 2) and run side by side;
- then the point-wise kernels of all problems run.

Each problem keeps its own time step and step count. A problem's results in
a batch are the ones it gets alone, bit for bit.

The reference has no batch API. The nearest form is one ``Simulation`` per
thread (python/src/bindings.cpp:336-337).
"""

from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

from . import native as N
from .problem import ProblemData
from .solver import Solver


class BatchMember(Solver):
    """A problem inside a batch: the ``Solver`` accessors (state, trace,
    energy, set_state before the first batched step) on a handle the batch
    owns. It cannot be advanced on its own."""

    def __init__(self, batch: "Batch", index: int, problem: ProblemData):
        self.problem = problem
        self._packed = None
        self._traces = problem.trace_list()
        self._batch = batch
        self.index = index
        h = N.lib().insem_cuda_batch_member(batch._h, index)
        if not h:
            N.check(N.ERR_INVALID)
        self._h = C.c_void_p(h)

    def close(self) -> None:
        self._h = None  # the batch owns the handle


class Batch:
    def __init__(self, device: int = 0, use_graphs: bool = True, check_finite: bool = True, tile_streams: int = 0):
        opts = N.Options(device, int(use_graphs), 0, 0, int(check_finite), int(tile_streams))
        h = C.c_void_p()
        N.check(N.lib().insem_cuda_batch_create(C.byref(opts), C.byref(h)))
        self._h = h
        self.device = device
        self.members: List[Optional[BatchMember]] = []

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            for m in self.members:
                if m is not None:
                    m._h = None
            N.lib().insem_cuda_batch_destroy(self._h)
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

    def add(self, problem: ProblemData) -> BatchMember:
        packed = problem.to_c()
        idx = C.c_int32()
        N.check(N.lib().insem_cuda_batch_add(self._h, packed.ref(), C.byref(idx)))
        m = BatchMember(self, idx.value, problem)
        self.members.append(m)
        return m

    def adopt(self, solver: Solver) -> BatchMember:
        """Moves an existing (not yet stepped by a batch) solver into the batch."""
        idx = C.c_int32()
        N.check(N.lib().insem_cuda_batch_adopt(self._h, solver._h, C.byref(idx)))
        solver._h = None  # owned by the batch now
        m = BatchMember(self, idx.value, solver.problem)
        self.members.append(m)
        return m

    def remove(self, member: BatchMember) -> None:
        N.check(N.lib().insem_cuda_batch_remove(self._h, member.index))
        member._h = None
        self.members[member.index] = None

    def advance(self, n_steps: int) -> None:
        N.check(N.lib().insem_cuda_batch_advance(self._h, int(n_steps)))

    def run(self) -> None:
        N.check(N.lib().insem_cuda_batch_run(self._h))

    def stream_layout(self):
        """(amplitude columns, sample-row columns) of the streamed steps of the
        current composition: active members in index order."""
        a, r = C.c_int32(), C.c_int32()
        N.check(N.lib().insem_cuda_batch_stream_layout(self._h, C.byref(a), C.byref(r)))
        return a.value, r.value

    def active_members(self) -> List["BatchMember"]:
        return [m for m in self.members if m is not None and m.step < m.n_steps]

    def advance_streamed(self, n_steps: int, amplitudes, rows_out=None) -> int:
        """n_steps batched steps (fewer if every member ends sooner) with
        per-step host I/O: ``amplitudes`` [n_steps, amp_cols] float32 in (None:
        the members' own source time functions), ``rows_out`` [n_steps,
        row_cols] float64 out (numpy arrays or pinned torch tensors).  A member
        with r steps left has valid rows for its first r steps.  Returns the
        steps done."""
        def ptr(x, ctype):
            if x is None:
                return None
            if hasattr(x, "data_ptr"):
                return C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ctype))
            return x.ctypes.data_as(C.POINTER(ctype))

        done = C.c_int32()
        N.check(N.lib().insem_cuda_batch_advance_streamed(self._h, int(n_steps), ptr(amplitudes, C.c_float),
                                                          ptr(rows_out, C.c_double), C.byref(done)))
        return done.value

    def profile(self, n_steps: int) -> Tuple[float, float]:
        """n steps with plain launches and CUDA events around each step's tile
        launches: (device ms of the tile launches, device ms of the steps)."""
        t, st = C.c_double(), C.c_double()
        N.check(N.lib().insem_cuda_batch_profile(self._h, int(n_steps), C.byref(t), C.byref(st)))
        return t.value, st.value

    @property
    def active(self) -> int:
        return int(N.lib().insem_cuda_batch_active(self._h))

    @property
    def steps_to_next_completion(self) -> int:
        return int(N.lib().insem_cuda_batch_steps_to_next_completion(self._h))

    @property
    def steps_to_completion(self) -> int:
        """Steps until every member is complete."""
        return int(N.lib().insem_cuda_batch_steps_to_completion(self._h))

    @property
    def last_advance_ms(self) -> float:
        return float(N.lib().insem_cuda_batch_last_advance_ms(self._h))

    @property
    def point_updates(self) -> int:
        return int(N.lib().insem_cuda_batch_point_updates(self._h))

    @property
    def kernels_per_step(self) -> int:
        return int(N.lib().insem_cuda_batch_kernels_per_step(self._h))
