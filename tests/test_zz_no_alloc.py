"""The allocation-free internal-forces entry point (collected last, so that a
run stopping at its first failure has run every other test before it).

insem_cuda_solver_internal_forces_noalloc serves callers that cannot let the
library allocate device memory: applications whose GPU memory is owned by
another allocator, and loops that cannot absorb cudaFree's wait for the whole
device. It computes what insem_cuda_solver_internal_forces computes, on
device arrays the caller passes, with its element-local scratch in a fixed
array inside the library. These tests check it against the allocating entry
point, bit for bit (the tolerance of every internal-forces test here), on two
calls in a row that reuse that array, and check that a domain too large for
the array is refused before any work is enqueued.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _noalloc(solver, domain, u_dev, f_dev, stream_handle):
    from insem_b200 import native as N

    return N.lib().insem_cuda_solver_internal_forces_noalloc(
        solver._h, int(domain), C.c_void_p(u_dev.data_ptr()), C.c_void_p(f_dev.data_ptr()),
        C.c_void_p(stream_handle) if stream_handle else None)


def test_noalloc_matches_allocating_entry_point_on_two_calls(pkg):
    import torch

    from insem_b200 import native as N

    z = golden("lay")  # coupled: elastic and acoustic domains, curved Quad9 cells
    prob = pkg.ProblemData.from_npz(z)
    rng = np.random.default_rng(11)
    side = torch.cuda.Stream()
    with pkg.Solver(prob) as s:
        # first call: the elastic domain on the legacy default stream; second
        # call, right after: the acoustic domain on another stream, over the
        # scratch the first call left behind
        order = sorted(range(len(prob.domains)), key=lambda i: -prob.domains[i].ncomp)
        for call, di in enumerate(order):
            d = prob.domains[di]
            u = rng.uniform(-1.0, 1.0, d.ncomp * d.n_global).astype(np.float32)
            want = s.internal_forces(di, u)
            u_dev = torch.from_numpy(u).cuda()
            f_dev = torch.full((d.ncomp * d.n_global,), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            handle = side.cuda_stream if call == 1 else 0
            assert _noalloc(s, di, u_dev, f_dev, handle) == N.OK, N.lib().insem_cuda_last_error()
            torch.cuda.synchronize()
            got = f_dev.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), np.asarray(want, np.float32).reshape(-1).view(np.uint32)), \
                (call, di)


def test_noalloc_refuses_a_domain_beyond_its_scratch(pkg):
    import torch

    from insem_b200 import cases as K
    from insem_b200 import native as N

    # 300 x 300 order-5 cells: the elastic domain needs 2 x ~76k x 36 floats,
    # more than the 4,194,304 the fixed array holds
    prob = K.build(K.config3(nx=300, n_steps=10, n_receivers=8), stable_dt=1e-5)
    di = next(i for i, d in enumerate(prob.domains) if d.medium == N.ELASTIC)
    d = prob.domains[di]
    assert d.ncomp * d.n_elements * prob.ngll ** 2 > (1 << 22)
    with pkg.Solver(prob) as s:
        u_dev = torch.zeros(d.ncomp * d.n_global, dtype=torch.float32, device="cuda")
        f_dev = torch.full_like(u_dev, 7.0)
        rc = _noalloc(s, di, u_dev, f_dev, 0)
        assert rc == N.ERR_UNSUPPORTED
        assert b"4194304" in N.lib().insem_cuda_last_error()
        torch.cuda.synchronize()
        assert bool(torch.all(f_dev == 7.0))  # nothing was enqueued


def test_noalloc_calls_leave_free_device_memory_unchanged(pkg):
    """The property the entry point exists for: on a freshly created solver,
    its first call and every later one change the device's free memory by
    nothing (no cudaMalloc, and no module the driver loads on first use)."""
    import torch

    from insem_b200 import native as N

    z = golden("bh1")  # axisymmetric m = 1: hanging-node rows, both media
    prob = pkg.ProblemData.from_npz(z)
    rng = np.random.default_rng(5)
    inputs = []
    for d in prob.domains:
        u = torch.from_numpy(rng.uniform(-1.0, 1.0, d.ncomp * d.n_global).astype(np.float32)).cuda()
        inputs.append((u, torch.empty_like(u)))
    with pkg.Solver(prob) as s:
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(3):
            for di, (u_dev, f_dev) in enumerate(inputs):
                assert _noalloc(s, di, u_dev, f_dev, 0) == N.OK, N.lib().insem_cuda_last_error()
            torch.cuda.synchronize()
            free, _ = torch.cuda.mem_get_info()
            assert free == free0, f"free device memory changed by {free0 - free} bytes"
