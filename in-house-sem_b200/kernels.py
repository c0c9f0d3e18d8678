"""Per-block kernel seam and DofMap seam through the C ABI.

``block_forces`` mirrors ``physics::{elastic,acoustic}_internal_forces``
(cpp/include/insem/physics/kernels.hpp:32-35): host arrays in, host arrays
out, only the block's elements of ``f_local`` written.  ``gather`` and
``assemble`` mirror ``DofMap::gather/assemble`` (dof_map.hpp:73-77).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N
from .problem import BlockData, DomainData, ProblemData, _f32, _f64, _i32


class BlockKernel:
    """One uploaded element block (kernel seam handle)."""

    def __init__(self, problem: ProblemData, block: BlockData, medium: int, device: int = 0):
        self._keep = []

        def ptr(a, ctype):
            if a is None or np.asarray(a).size == 0:
                return C.cast(None, C.POINTER(ctype))
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(ctype))

        basis = N.Basis(problem.ngll, ptr(_f32(problem.D), C.c_float), ptr(_f32(problem.Dj), C.c_float),
                        ptr(_f32(problem.w2), C.c_float))
        blk = N.Block(block.kind, block.azimuthal_order, block.n_elements, ptr(_i32(block.elements), C.c_int32),
                      ptr(_f32(block.metric), C.c_float), ptr(_f32(block.coef0), C.c_float),
                      ptr(_f32(block.coef1), C.c_float), ptr(_f32(block.wr), C.c_float),
                      ptr(_f32(block.hoop), C.c_float), ptr(_f32(block.r), C.c_float),
                      ptr(np.ascontiguousarray(block.axial, np.uint8), C.c_uint8))
        h = C.c_void_p()
        N.check(N.lib().insem_cuda_block_create(C.byref(basis), C.byref(blk), medium, device, C.byref(h)))
        self._h = h

    def forces(self, n_local_elements: int, u_local: np.ndarray, f_local: np.ndarray) -> None:
        """f_local[block elements] = -K u_local (host arrays, f_local updated in place)."""
        assert u_local.dtype == np.float32 and f_local.dtype == np.float32 and f_local.flags.c_contiguous
        u_local = np.ascontiguousarray(u_local)
        N.check(N.lib().insem_cuda_block_forces_host(self._h, n_local_elements, u_local.ctypes.data_as(N.f32p),
                                                     f_local.ctypes.data_as(N.f32p)))

    def forces_device(self, n_local_elements: int, u_ptr: int, f_ptr: int, stream: int = 0) -> None:
        """Asynchronous variant on device pointers (e.g. torch tensors' data_ptr())."""
        N.check(N.lib().insem_cuda_block_forces(self._h, n_local_elements, C.c_void_p(u_ptr), C.c_void_p(f_ptr),
                                                C.c_void_p(stream)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().insem_cuda_block_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def block_forces(problem: ProblemData, domain: int, block: int, u_local: np.ndarray, device: int = 0) -> np.ndarray:
    """f_local of one block for an element-local field of the whole domain."""
    d = problem.domains[domain]
    f = np.zeros(d.ncomp * d.n_elements * problem.ngll ** 2, np.float32)
    k = BlockKernel(problem, d.blocks[block], d.medium, device)
    try:
        k.forces(d.n_elements, np.asarray(u_local, np.float32).ravel(), f)
    finally:
        k.close()
    return f


class DofMapKernel:
    """One uploaded DofMap (gather/assemble seam handle)."""

    def __init__(self, ngll: int, d: DomainData, device: int = 0):
        self._keep = []

        def ptr(a, ctype):
            if a is None or np.asarray(a).size == 0:
                return C.cast(None, C.POINTER(ctype))
            self._keep.append(a)
            return a.ctypes.data_as(C.POINTER(ctype))

        weighted = d.n_rows > 0 and d.t_weights.size > 0
        dm = N.DofMap(ngll, d.n_elements, d.n_global, ptr(_i32(d.l2g), C.c_int32), d.n_rows,
                      ptr(_i32(d.row_offsets), C.c_int32), ptr(_i32(d.row_dofs), C.c_int32),
                      ptr(_f64(d.row_weights), C.c_double), ptr(_i32(d.t_offsets), C.c_int32),
                      ptr(_i32(d.t_slots), C.c_int32),
                      ptr(_f64(d.t_weights), C.c_double) if weighted else C.cast(None, N.f64p))
        h = C.c_void_p()
        N.check(N.lib().insem_cuda_dofmap_create(C.byref(dm), device, C.byref(h)))
        self._h = h
        self.d = d
        self.npe = ngll * ngll

    def gather_device(self, ncomp: int, g_ptr: int, l_ptr: int, stream: int = 0) -> None:
        N.check(N.lib().insem_cuda_gather(self._h, ncomp, C.c_void_p(g_ptr), C.c_void_p(l_ptr), C.c_void_p(stream)))

    def assemble_device(self, ncomp: int, l_ptr: int, g_ptr: int, stream: int = 0) -> None:
        N.check(N.lib().insem_cuda_assemble(self._h, ncomp, C.c_void_p(l_ptr), C.c_void_p(g_ptr),
                                            C.c_void_p(stream)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().insem_cuda_dofmap_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
