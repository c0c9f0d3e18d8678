"""ctypes binding of the C ABI in ``include/insem_cuda.h``.

The shared library ``lib/libinsem_cuda.so`` is built in-tree (``build.py``).
Loading fails loudly when it is missing: there is no CPU fallback for any
entry point of this package.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libinsem_cuda.so"

OK = 0
ERR_INVALID = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_STATE = 4
ERR_NOMEM = 5
ERR_NONFINITE = 6
ERR_TIMEOUT = 7

ACOUSTIC, ELASTIC = 0, 1
RECT, AFFINE, CURVED, AXISYM = 0, 1, 2, 3
QUANTITIES = {"displacement": 0, "velocity": 1, "acceleration": 2, "pressure": 3, "particle_velocity": 4}

i32p = C.POINTER(C.c_int32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
u8p = C.POINTER(C.c_uint8)


class InsemError(RuntimeError):
    """Error reported by the backend (the reference raises insem.InsemError for the same conditions)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class Basis(C.Structure):
    _fields_ = [("ngll", C.c_int32), ("D", f32p), ("Dj", f32p), ("w2", f32p)]


class Block(C.Structure):
    _fields_ = [("kind", C.c_int32), ("azimuthal_order", C.c_int32), ("n_elements", C.c_int32),
                ("elements", i32p), ("metric", f32p), ("coef0", f32p), ("coef1", f32p),
                ("wr", f32p), ("hoop", f32p), ("r", f32p), ("axial", u8p)]


class DofMap(C.Structure):
    _fields_ = [("ngll", C.c_int32), ("n_elements", C.c_int32), ("n_global", C.c_int32), ("l2g", i32p),
                ("n_rows", C.c_int32), ("row_offsets", i32p), ("row_dofs", i32p), ("row_weights", f64p),
                ("t_offsets", i32p), ("t_slots", i32p), ("t_weights", f64p)]


class Domain(C.Structure):
    _fields_ = [("medium", C.c_int32), ("ncomp", C.c_int32), ("azimuthal_order", C.c_int32), ("dofs", DofMap),
                ("n_blocks", C.c_int32), ("blocks", C.POINTER(Block)), ("mass", f32p), ("inv_mass", f32p),
                ("n_absorbing", C.c_int32), ("absorbing_points", i32p), ("absorbing_coef", f32p),
                ("n_dirichlet", C.c_int32), ("dirichlet_points", i32p), ("n_axis", C.c_int32),
                ("axis_points", i32p), ("n_axis_components", C.c_int32), ("axis_components", i32p)]


class Coupling(C.Structure):
    _fields_ = [("n", C.c_int32), ("fluid_points", i32p), ("solid_points", i32p), ("cx", f32p), ("cz", f32p)]


class Stf(C.Structure):
    _fields_ = [("kind", C.c_int32), ("f0", C.c_double), ("t0", C.c_double), ("amplitude", C.c_double),
                ("n_samples", C.c_int32), ("samples", f64p), ("sample_dt", C.c_double)]


class Source(C.Structure):
    _fields_ = [("domain", C.c_int32), ("n_points", C.c_int32), ("points", i32p), ("coef", f32p), ("stf", Stf)]


class Receiver(C.Structure):
    _fields_ = [("domain", C.c_int32), ("n_points", C.c_int32), ("points", i32p), ("value", f32p),
                ("d_dx", f32p), ("d_dz", f32p), ("rho", C.c_double), ("n_quantities", C.c_int32),
                ("quantities", i32p)]


class Problem(C.Structure):
    _fields_ = [("basis", Basis), ("n_domains", C.c_int32), ("domains", C.POINTER(Domain)),
                ("coupling", Coupling), ("n_sources", C.c_int32), ("sources", C.POINTER(Source)),
                ("n_receivers", C.c_int32), ("receivers", C.POINTER(Receiver)), ("dt", C.c_double),
                ("n_steps", C.c_int32), ("record_every", C.c_int32), ("energy_every", C.c_int32)]


class Time(C.Structure):
    """insem_cuda_time: the reference's TimeConfig (dt, safety, n_steps, duration)."""
    _fields_ = [("dt", C.c_double), ("safety", C.c_double), ("n_steps", C.c_int32), ("duration", C.c_double)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("use_graphs", C.c_int32), ("path", C.c_int32),
                ("tile_elements", C.c_int32), ("check_finite", C.c_int32), ("tile_streams", C.c_int32)]


_lib = None


def lib() -> C.CDLL:
    """The loaded backend library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise InsemError(ERR_CUDA, f"CUDA backend library missing: {LIB_PATH} (run build.py)")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        sig = {
            "insem_cuda_last_error": (C.c_char_p, []),
            "insem_cuda_version": (C.c_char_p, []),
            "insem_cuda_mem_info": (C.c_int, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
            "insem_cuda_block_create": (C.c_int, [C.POINTER(Basis), C.POINTER(Block), C.c_int32, C.c_int32, C.POINTER(vp)]),
            "insem_cuda_block_destroy": (None, [vp]),
            "insem_cuda_block_forces": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
            "insem_cuda_block_forces_host": (C.c_int, [vp, C.c_int32, f32p, f32p]),
            "insem_cuda_dofmap_create": (C.c_int, [C.POINTER(DofMap), C.c_int32, C.POINTER(vp)]),
            "insem_cuda_dofmap_destroy": (None, [vp]),
            "insem_cuda_gather": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
            "insem_cuda_assemble": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
            "insem_cuda_solver_create": (C.c_int, [C.POINTER(Problem), C.POINTER(Options), C.POINTER(vp)]),
            "insem_cuda_solver_create_timed": (C.c_int, [C.POINTER(Problem), C.POINTER(Time), C.POINTER(Options),
                                                         C.POINTER(vp)]),
            "insem_cuda_solver_stable_dt": (C.c_double, [vp]),
            "insem_cuda_solver_destroy": (None, [vp]),
            "insem_cuda_solver_set_state": (C.c_int, [vp, C.c_int32, f64p, f64p]),
            "insem_cuda_solver_advance": (C.c_int, [vp, C.c_int32]),
            "insem_cuda_solver_run": (C.c_int, [vp]),
            "insem_cuda_solver_step": (C.c_int32, [vp]),
            "insem_cuda_solver_status": (C.c_int32, [vp]),
            "insem_cuda_solver_n_steps": (C.c_int32, [vp]),
            "insem_cuda_solver_dt": (C.c_double, [vp]),
            "insem_cuda_solver_n_samples": (C.c_int32, [vp]),
            "insem_cuda_solver_n_traces": (C.c_int32, [vp]),
            "insem_cuda_solver_trace_ncomp": (C.c_int32, [vp, C.c_int32]),
            "insem_cuda_solver_trace": (C.c_int, [vp, C.c_int32, f64p]),
            "insem_cuda_solver_times": (C.c_int, [vp, f64p]),
            "insem_cuda_solver_energy": (C.c_int, [vp, f64p, C.c_int32, i32p]),
            "insem_cuda_solver_state": (C.c_int, [vp, C.c_int32, f64p, f64p, f64p]),
            "insem_cuda_solver_set_snapshots": (C.c_int, [vp, C.c_int32, C.c_int32, i32p]),
            "insem_cuda_solver_n_snapshots": (C.c_int32, [vp]),
            "insem_cuda_solver_n_snapshot_fields": (C.c_int32, [vp]),
            "insem_cuda_solver_snapshot_field": (C.c_int, [vp, C.c_int32, i32p, i32p, i32p, C.POINTER(C.c_int64)]),
            "insem_cuda_solver_snapshot": (C.c_int, [vp, C.c_int32, f32p]),
            "insem_cuda_solver_snapshot_times": (C.c_int, [vp, f64p]),
            "insem_cuda_solver_last_advance_ms": (C.c_double, [vp]),
            "insem_cuda_solver_internal_forces": (C.c_int, [vp, C.c_int32, f32p, f32p]),
            "insem_cuda_solver_internal_forces_noalloc": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
            "insem_cuda_stable_dt": (C.c_int, [C.POINTER(Problem), C.c_int32, f64p]),
            "insem_cuda_solver_advance_streamed": (C.c_int, [vp, C.c_int32, f32p, f64p, i32p]),
            "insem_cuda_solver_n_columns": (C.c_int32, [vp]),
            "insem_cuda_solver_kernels_per_step": (C.c_int32, [vp]),
            "insem_cuda_batch_create": (C.c_int, [C.POINTER(Options), C.POINTER(vp)]),
            "insem_cuda_batch_destroy": (None, [vp]),
            "insem_cuda_batch_add": (C.c_int, [vp, C.POINTER(Problem), i32p]),
            "insem_cuda_batch_adopt": (C.c_int, [vp, vp, i32p]),
            "insem_cuda_solver_prepare_for_batch": (C.c_int, [vp]),
            "insem_cuda_batch_advance": (C.c_int, [vp, C.c_int32]),
            "insem_cuda_batch_run": (C.c_int, [vp]),
            "insem_cuda_batch_remove": (C.c_int, [vp, C.c_int32]),
            "insem_cuda_batch_member": (vp, [vp, C.c_int32]),
            "insem_cuda_batch_advance_streamed": (C.c_int, [vp, C.c_int32, f32p, f64p, i32p]),
            "insem_cuda_batch_stream_layout": (C.c_int, [vp, i32p, i32p]),
            "insem_cuda_batch_profile": (C.c_int, [vp, C.c_int32, f64p, f64p]),
            "insem_cuda_solver_point_classes": (C.c_int, [vp, C.c_int32, i32p, i32p]),
            "insem_cuda_set_tile_elements": (C.c_int, [C.c_int32] * 5),
            "insem_cuda_tile_elements": (C.c_int32, [C.c_int32] * 5),
            "insem_cuda_solver_tile_elements": (C.c_int32, [vp, C.c_int32]),
            "insem_cuda_batch_size": (C.c_int32, [vp]),
            "insem_cuda_batch_active": (C.c_int32, [vp]),
            "insem_cuda_batch_steps_to_next_completion": (C.c_int32, [vp]),
            "insem_cuda_batch_steps_to_completion": (C.c_int32, [vp]),
            "insem_cuda_batch_last_advance_ms": (C.c_double, [vp]),
            "insem_cuda_batch_point_updates": (C.c_int64, [vp]),
            "insem_cuda_batch_kernels_per_step": (C.c_int32, [vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    """Names declared in the header that the library must export."""
    header = PKG.parent / "include" / "insem_cuda.h"
    import re

    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(insem_cuda_\w+)\s*\(", header.read_text(), re.M)
    return sorted(set(names))


def check(rc: int) -> None:
    """Raises InsemError for a non-zero status, with the library's message."""
    if rc != OK:
        msg = lib().insem_cuda_last_error().decode(errors="replace")
        raise InsemError(rc, msg or f"insem_cuda error {rc}")
