"""Host-side checks of the C ABI (CPU only, no compute calls)."""

from __future__ import annotations

import ctypes as C
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden


def test_library_exports_every_declared_symbol(pkg):
    from insem_b200 import native

    declared = native.exported_symbols()
    assert len(declared) >= 28
    L = C.CDLL(str(native.LIB_PATH))
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(native.LIB_PATH)], capture_output=True, text=True).stdout
    for n in declared:
        assert f" T {n}" in out, n


def test_version_and_error_state(pkg):
    L = pkg.lib()
    assert L.insem_cuda_version().startswith(b"insem-b200")
    assert L.insem_cuda_last_error() is not None


def test_missing_library_fails_loudly(pkg, monkeypatch, tmp_path):
    from insem_b200 import native

    monkeypatch.setattr(native, "_lib", None)
    monkeypatch.setattr(native, "LIB_PATH", tmp_path / "missing.so")
    with pytest.raises(native.InsemError, match="CUDA backend library missing"):
        native.lib()


def test_struct_layout_matches_header(pkg):
    """Sizes of the ctypes mirrors equal the C structs (checked with the host compiler)."""
    from insem_b200 import native as N

    src = r'''
#include <stdio.h>
#include "insem_cuda.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(insem_cuda_basis),
         sizeof(insem_cuda_block), sizeof(insem_cuda_dofmap), sizeof(insem_cuda_domain), sizeof(insem_cuda_coupling),
         sizeof(insem_cuda_stf), sizeof(insem_cuda_source), sizeof(insem_cuda_receiver), sizeof(insem_cuda_problem),
         sizeof(insem_cuda_options), offsetof(insem_cuda_problem, dt), sizeof(insem_cuda_time),
         offsetof(insem_cuda_time, n_steps), offsetof(insem_cuda_time, duration));
  return 0;
}
'''
    import tempfile, os

    with tempfile.TemporaryDirectory() as d:
        cfile = os.path.join(d, "sz.c")
        open(cfile, "w").write("#include <stddef.h>\n" + src)
        exe = os.path.join(d, "sz")
        subprocess.run(["gcc", "-I", str(REPO / "include"), cfile, "-o", exe], check=True)
        sizes = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    ours = [C.sizeof(t) for t in (N.Basis, N.Block, N.DofMap, N.Domain, N.Coupling, N.Stf, N.Source,
                                  N.Receiver, N.Problem, N.Options)] + [N.Problem.dt.offset, C.sizeof(N.Time),
                                                                        N.Time.n_steps.offset, N.Time.duration.offset]
    assert sizes == ours


def test_problem_round_trip(pkg):
    z = golden("bh1")
    prob = pkg.ProblemData.from_npz(z)
    packed = prob.to_c()
    s = packed.struct
    assert s.n_domains == len(prob.domains) == 2
    assert s.basis.ngll == prob.ngll
    d1 = prob.domains[1]
    assert s.domains[1].dofs.n_global == d1.n_global
    assert s.domains[1].dofs.n_rows == d1.n_rows > 0
    assert s.domains[1].blocks[0].azimuthal_order == 1
    assert s.n_receivers == len(prob.receivers)
    assert prob.trace_list()[0] == ("p1", "pressure")
    assert prob.algorithmic_bytes_per_step() > 0


def test_algorithmic_bytes_c1(pkg):
    prob = pkg.ProblemData.from_npz(golden("c1"))
    # 16,641 points x 20 B + 1024 Rect acoustic elements x (4*25 + 12 + 4*25) B
    assert prob.algorithmic_bytes_per_step() == 16641 * 20 + 1024 * (100 + 12 + 100)


def test_timed_constructor_rejects_null_arguments(pkg):
    """Argument checks of insem_cuda_solver_create_timed come before any device work."""
    from insem_b200 import native as N

    L = pkg.lib()
    t = N.Time(0.0, 0.8, 0, 1e-3)
    h = C.c_void_p()
    assert L.insem_cuda_solver_create_timed(None, C.byref(t), None, C.byref(h)) == N.ERR_INVALID
    assert b"null" in L.insem_cuda_last_error()
    assert not h.value
    assert L.insem_cuda_solver_stable_dt(None) == 0.0
