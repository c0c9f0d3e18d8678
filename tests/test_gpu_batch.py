"""Batched solves on the GPU: every problem's results in a batch equal the
reference's (golden fixtures) and equal the same problem solved alone, bit
for bit, whatever the mix (ngll, geometry kinds, media, azimuthal orders,
step counts) and the step chunking."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import RUN_CASES, golden
import golden_io as G

pytestmark = pytest.mark.gpu


def _init_state(member, prob, z):
    for di in range(len(prob.domains)):
        if f"init.d{di}.u" in z.files and (np.any(z[f"init.d{di}.u"]) or np.any(z[f"init.d{di}.v"])):
            member.set_state(prob.media[di], z[f"init.d{di}.u"].astype(np.float64),
                             z[f"init.d{di}.v"].astype(np.float64))


def _check_golden(case, prob, s, z):
    assert s.step == prob.n_steps
    assert np.array_equal(s.times, z["run.times"])
    for name, q in prob.trace_list():
        gold = z[f"run.trace.{name}.{q}"]
        got = s.trace(name, q)
        assert np.array_equal(got, gold), f"{case} {name}/{q}: rel L2 {G.rel_l2(got, gold):.3e}"
    for di in range(len(prob.domains)):
        for key, arr in zip("uva", s.state(prob.media[di])):
            gold = z[f"run.d{di}.{key}"].astype(np.float64).reshape(arr.shape)
            assert np.array_equal(arr, gold), f"{case} d{di} {key}"
    e, ge = s.energy, z["run.energy"]
    assert e.shape == ge.shape
    if ge.size:
        assert np.array_equal(e[:, 0], ge[:, 0])
        assert np.abs(e[:, 1:] - ge[:, 1:]).max() <= 1e-9 * np.abs(ge[:, 1:]).max()


@pytest.mark.parametrize("graphs,streams", [(True, 0), (False, 0), (True, 1), (True, 8)])
def test_batch_of_all_cases_matches_reference(pkg, graphs, streams):
    """Every case in one batch; the tile classes on the default number of
    streams, on one stream and on eight (results do not depend on it)."""
    from insem_b200 import Batch

    with Batch(use_graphs=graphs, tile_streams=streams) as b:
        entries = []
        for case in RUN_CASES:
            z = golden(case)
            prob = pkg.ProblemData.from_npz(z)
            m = b.add(prob)
            _init_state(m, prob, z)
            entries.append((case, prob, m, z))
        b.advance(5)
        assert b.active == len(RUN_CASES)
        if graphs:
            assert b.kernels_per_step >= 3
        b.run()
        assert b.active == 0
        for case, prob, m, z in entries:
            _check_golden(case, prob, m, z)


def test_same_result_alone_and_in_mix(pkg):
    """Two copies of a layered ocean-bottom model, a borehole and the README
    model in one batch, stepped in uneven chunks, against each solved alone."""
    from insem_b200 import Batch, cases as K

    probs = [K.build(K.config3(nx=40, n_steps=90, n_receivers=32)), pkg.ProblemData.from_npz(golden("bh1")),
             K.build(K.config3(nx=40, n_steps=60, n_receivers=8)), pkg.ProblemData.from_npz(golden("c1"))]
    alone = []
    for p in probs:
        with pkg.Solver(p) as s:
            s.run()
            alone.append(([s.trace(n, q) for n, q in p.trace_list()], [s.state(md) for md in p.media]))
    with Batch() as b:
        ms = [b.add(p) for p in probs]
        for k in (1, 2, 7, 13):
            b.advance(k)
        b.run()
        for p, m, (traces, states) in zip(probs, ms, alone):
            assert m.step == p.n_steps
            for (n, q), t in zip(p.trace_list(), traces):
                assert np.array_equal(m.trace(n, q), t), (n, q)
            for md, st in zip(p.media, states):
                for a, b2 in zip(m.state(md), st):
                    assert np.array_equal(a, b2), md


def test_member_is_not_advanced_alone(pkg):
    from insem_b200 import Batch, InsemError

    prob = pkg.ProblemData.from_npz(golden("c1"))
    with Batch() as b:
        m = b.add(prob)
        b.advance(2)
        with pytest.raises(InsemError):
            m.advance(1)
        assert m.step == 2
        b.remove(m)
        assert b.active == 0


def test_adopted_solver_continues_bitwise(pkg):
    """A solver advanced alone for a few steps, then moved into a batch."""
    from insem_b200 import Batch

    z = golden("lay")
    prob = pkg.ProblemData.from_npz(z)
    s = pkg.Solver(prob)
    _init_state(s, prob, z)
    s.advance(11)
    with Batch() as b:
        m = b.adopt(s)
        b.run()
        _check_golden("lay", prob, m, z)


def test_batch_streamed_rows_match_reference(pkg):
    """Streamed batched steps (amplitudes in, sample rows out, every step) give
    the reference's samples, member by member, across completions."""
    from insem_b200 import Batch
    from insem_b200.stf import amplitudes

    with Batch() as b:
        ref = {}
        for case in ("c1", "lay", "bh1"):
            z = golden(case)
            prob = pkg.ProblemData.from_npz(z)
            m = b.add(prob)
            _init_state(m, prob, z)
            full = np.concatenate([z[f"run.trace.{n}.{q}"] for n, q in prob.trace_list()], axis=1)
            ref[m.index] = (prob, full)
        b.advance(3)
        checked = 0
        while b.active:
            amp_cols, row_cols = b.stream_layout()
            act = b.active_members()
            k = min(b.steps_to_next_completion, 37)
            first = {m.index: m.step + 1 for m in act}
            amp = np.concatenate([amplitudes(ref[m.index][0], first[m.index], k) for m in act], axis=1)
            amp = np.ascontiguousarray(amp, np.float32)
            assert amp.shape[1] == amp_cols
            rows = np.zeros((k, row_cols))
            got = b.advance_streamed(k, amp, rows)
            assert got == k
            col = 0
            for m in act:
                prob, full = ref[m.index]
                nc = full.shape[1]
                for j in range(got):
                    s = first[m.index] + j
                    assert np.array_equal(rows[j, col:col + nc], full[s // prob.record_every]), (m.index, s)
                    checked += 1
                col += nc
            assert col == row_cols
        assert checked > 0
