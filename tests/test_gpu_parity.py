"""CUDA path vs the reference's own outputs (golden fixtures made from the
reference build): per-block force vectors, gather, assemble and internal
forces bit for bit; full-run receiver traces, sample times and final fields
bit for bit; energy samples to 1e-9 relative (FP64 reductions in a different
order); the stable time step to 1e-6 relative."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import BLK_CASES, RUN_CASES, golden
import golden_io as G

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32)


@pytest.mark.parametrize("case", RUN_CASES + BLK_CASES)
def test_block_forces_bitwise(pkg, case):
    from insem_b200 import kernels

    z = golden(case)
    n = 0
    for prefix, prob in G.sub_problems(pkg, z):
        for di, d in enumerate(prob.domains):
            u = G.block_input(d, di)
            for bi in range(len(d.blocks)):
                f = kernels.block_forces(prob, di, bi, u)
                gold = z[f"{prefix}gold.d{di}.b{bi}.f_local"]
                assert np.array_equal(bits(f), bits(gold)), f"{case} {prefix} d{di} b{bi}"
                n += 1
    assert n > 0


@pytest.mark.parametrize("case", RUN_CASES + BLK_CASES)
def test_gather_assemble_bitwise(pkg, case):
    import torch
    from insem_b200 import kernels

    z = golden(case)
    for prefix, prob in G.sub_problems(pkg, z):
        for di, d in enumerate(prob.domains):
            k = kernels.DofMapKernel(prob.ngll, d)
            g = torch.from_numpy(G.gather_input(d, di)).cuda()
            loc = torch.empty(d.ncomp * d.l2g.size, dtype=torch.float32, device="cuda")
            k.gather_device(d.ncomp, g.data_ptr(), loc.data_ptr())
            fl = torch.from_numpy(G.assemble_input(d, di)).cuda()
            glob = torch.empty(d.ncomp * d.n_global, dtype=torch.float32, device="cuda")
            k.assemble_device(d.ncomp, fl.data_ptr(), glob.data_ptr())
            torch.cuda.synchronize()
            assert np.array_equal(bits(loc.cpu().numpy()), bits(z[f"{prefix}gold.d{di}.gather"]))
            assert np.array_equal(bits(glob.cpu().numpy()), bits(z[f"{prefix}gold.d{di}.assemble"]))
            k.close()


@pytest.mark.parametrize("case", RUN_CASES + BLK_CASES)
def test_internal_forces_bitwise(pkg, case):
    z = golden(case)
    for prefix, prob in G.sub_problems(pkg, z):
        with pkg.Solver(prob) as s:
            for di, d in enumerate(prob.domains):
                f = s.internal_forces(di, G.forces_input(d, di))
                assert np.array_equal(bits(f), bits(z[f"{prefix}gold.d{di}.internal_forces"]))


def run_case(pkg, z, **opts):
    prob = pkg.ProblemData.from_npz(z)
    s = pkg.Solver(prob, **opts)
    for di, d in enumerate(prob.domains):
        if f"init.d{di}.u" in z.files and (np.any(z[f"init.d{di}.u"]) or np.any(z[f"init.d{di}.v"])):
            s.set_state(prob.media[di], z[f"init.d{di}.u"].astype(np.float64), z[f"init.d{di}.v"].astype(np.float64))
    s.advance(int(z["run.advance_first"]))
    s.run()
    return prob, s


@pytest.mark.parametrize("path", [0, 1], ids=["tiled", "plain"])
@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", RUN_CASES)
def test_run_bitwise(pkg, case, graphs, path):
    z = golden(case)
    prob, s = run_case(pkg, z, use_graphs=graphs, path=path)
    with s:
        assert s.step == prob.n_steps
        assert np.array_equal(s.times, z["run.times"])
        for name, q in prob.trace_list():
            gold = z[f"run.trace.{name}.{q}"]
            got = s.trace(name, q)
            assert got.shape == gold.shape
            assert np.array_equal(got, gold), f"{case} {name}/{q}: rel L2 {G.rel_l2(got, gold):.3e}"
        for di in range(len(prob.domains)):
            u, v, a = s.state(prob.media[di])
            for key, arr in (("u", u), ("v", v), ("a", a)):
                gold = z[f"run.d{di}.{key}"].astype(np.float64).reshape(arr.shape)
                assert np.array_equal(arr, gold), f"{case} d{di} {key}"
        e = s.energy
        ge = z["run.energy"]
        assert e.shape == ge.shape
        if ge.size:
            assert np.array_equal(e[:, 0], ge[:, 0])
            scale = np.abs(ge[:, 1:]).max()
            assert np.abs(e[:, 1:] - ge[:, 1:]).max() <= 1e-9 * scale


@pytest.mark.parametrize("case", ["c1", "bh0", "lay", "box"])
def test_stable_dt(pkg, case):
    from insem_b200.solver import estimate_stable_dt

    z = golden(case)
    prob = pkg.ProblemData.from_npz(z)
    dt = estimate_stable_dt(prob)
    assert abs(dt - prob.stable_dt) <= 1e-6 * prob.stable_dt, (dt, prob.stable_dt)


@pytest.mark.parametrize("case", ["c1", "lay", "bh1"])
def test_streamed_advance_matches_traces(pkg, case):
    """Per-step amplitudes in / sample rows out give the same samples as the plain run."""
    from insem_b200.stf import amplitudes

    z = golden(case)
    prob = pkg.ProblemData.from_npz(z)
    with pkg.Solver(prob) as s:
        s.advance(3)
        n = prob.n_steps - 3
        amp = np.ascontiguousarray(amplitudes(prob, 4, n))
        rows = np.zeros((n // prob.record_every + 1, s.n_columns))
        got = s.advance_streamed(n, amp, rows)
        assert s.step == prob.n_steps
        assert s.kernels_per_step >= 3
    cols = []
    for name, q in prob.trace_list():
        cols.append(z[f"run.trace.{name}.{q}"])
    full = np.concatenate(cols, axis=1)
    first = 3 // prob.record_every + 1
    assert np.array_equal(rows[:got], full[first:first + got])


@pytest.mark.parametrize("nx", [48, 96])
def test_tiled_matches_plain_multi_tile(pkg, nx):
    """The layered ocean-bottom model at a size with many tiles per block (and
    padding points between tile ranges): tiled and plain paths agree bit for
    bit on traces and fields, and the finite check over the padded device
    arrays passes."""
    from insem_b200 import cases as K

    model = K.config3(nx=nx, n_steps=150, n_receivers=64)
    prob = K.build(model)
    with pkg.Solver(prob, path=0) as st, pkg.Solver(prob, path=1) as sp:
        st.advance(7)
        sp.advance(7)
        st.run()
        sp.run()
        for name, q in prob.trace_list():
            assert np.array_equal(st.trace(name, q), sp.trace(name, q)), f"{name}/{q}"
        for medium in prob.media:
            for a, b in zip(st.state(medium), sp.state(medium)):
                assert np.array_equal(a, b), medium
        et, ep = st.energy, sp.energy
        assert et.shape == ep.shape
        if ep.size:
            assert np.array_equal(et[:, 0], ep[:, 0])
            assert np.abs(et[:, 1:] - ep[:, 1:]).max() <= 1e-9 * np.abs(ep[:, 1:]).max()


@pytest.mark.parametrize("te", [3, 11, 64])
@pytest.mark.parametrize("case", ["lay", "bh1"])
def test_tile_size_does_not_change_results(pkg, case, te):
    """Any elements-per-tile (CTA size) gives the reference's bits."""
    z = golden(case)
    prob, s = run_case(pkg, z, tile_elements=te)
    with s:
        for name, q in prob.trace_list():
            assert np.array_equal(s.trace(name, q), z[f"run.trace.{name}.{q}"]), (case, te, name, q)
        for di in range(len(prob.domains)):
            u, v, a = s.state(prob.media[di])
            assert np.array_equal(u, z[f"run.d{di}.u"].astype(np.float64).reshape(u.shape))


def test_autotuner_registers_a_measured_choice(pkg):
    from insem_b200 import autotune

    prob = pkg.ProblemData.from_npz(golden("bh0"))
    keys = autotune.classes_of(prob)
    try:
        table = autotune.tune([prob], steps=5)
        assert set(table) == set(keys)
        for k, v in table.items():
            assert v["te"] in v["timings"] and autotune.current(k) == v["te"]
        with pkg.Solver(prob) as s:
            assert [s_te for s_te in (N_te(s, i) for i in range(len(prob.domains)))] == [table[k]["te"] for k in keys]
    finally:
        for k in keys:
            autotune.register(k, 0)


def N_te(s, domain):
    from insem_b200 import native as N

    return int(N.lib().insem_cuda_solver_tile_elements(s._h, domain))
