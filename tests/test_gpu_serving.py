"""Serving on the GPU: requests that arrive while others run join the running
batch; each request's streamed traces equal its solo run, bit for bit (the
same result alone and in the mix)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_stream():
    from insem_b200 import serving as S

    stream = S.request_stream(rate=300.0, window=1.0, time_scale=0.004, max_requests=14)
    for r in stream:
        if r.kind.startswith("cartesian"):
            r.spec["elements"] = min(r.spec["elements"], 5000.0)
    return stream


def _solo_traces(req):
    from insem_b200 import Solver, cases as K, serving as S

    model, arrays, _ = S.setup_request(req)
    prob = K.build_from_arrays(model, arrays)
    with Solver(prob) as s:
        s.run()
        return np.concatenate([s.trace_by_index(t) for t in range(len(prob.trace_list()))], axis=1)


def test_served_results_equal_solo_runs(pkg):
    from insem_b200 import serving as S

    stream = _small_stream()
    assert len({r.kind for r in stream}) >= 3
    recs = S.Server(chunk_steps=7).run(stream)
    summ = S.summarize(recs)
    assert summ["completed"] == len(stream)
    assert np.isfinite(summ["p99_ms_from_admission"]) and summ["value"] > 0
    for r in stream:
        rec = recs[r.rid]
        solo = _solo_traces(r)
        assert rec.traces.shape == solo.shape, (r.rid, r.kind)
        assert np.array_equal(rec.traces, solo), (r.rid, r.kind)


def test_admission_keeps_the_hbm_budget(pkg):
    """With an HBM budget of the largest request's footprint, the requests
    running at any admission never exceed the budget together, and the
    largest request runs alone."""
    from insem_b200 import serving as S

    stream = _small_stream()[:5]
    budget = max(S._stage_host(r)[3] for r in stream)
    recs = S.Server(hbm_budget=budget, chunk_steps=16).run(stream, keep_traces=False)
    done = list(recs.values())
    assert all(np.isfinite(r.completed) and r.status == "done" for r in done)
    for b in done:
        running = [r for r in done if r.admitted <= b.admitted < r.completed]
        assert sum(r.device_bytes for r in running) <= budget, (b.rid, [r.rid for r in running])
    big = max(done, key=lambda r: r.device_bytes)
    assert big.device_bytes == budget
    assert not [r.rid for r in done if r is not big and r.admitted < big.completed and big.admitted < r.completed]


def test_plain_server_runs_the_same_stream(pkg):
    from insem_b200 import serving as S

    stream = _small_stream()[:4]
    recs = S.serve_plain(stream, keep_traces=True)
    for r in stream:
        assert np.array_equal(recs[r.rid].traces, _solo_traces(r))


def test_timed_constructor_matches_two_step_route(pkg):
    """One device construction with the stable time step estimated inside
    (solver.cpp:131-144) gives the dt, step count and traces of
    stable-dt estimate + construction, bit for bit; a dt above the limit is
    rejected as in the reference."""
    from insem_b200 import Solver, cases as K, native as N, serving as S

    stream = _small_stream()
    seen = set()
    for r in stream:
        if r.kind in seen:
            continue
        seen.add(r.kind)
        model, arrays, _ = S.setup_request(r)
        prob_a = K.build_from_arrays(model, arrays)
        with Solver(prob_a) as a:
            a.run()
            ta = np.concatenate([a.trace_by_index(t) for t in range(len(prob_a.trace_list()))], axis=1)
        prob_b, b = K.build_solver_from_arrays(model, arrays)
        with b:
            assert prob_b.stable_dt == prob_a.stable_dt, r.kind
            assert b.dt == prob_a.dt and b.n_steps == prob_a.n_steps, r.kind
            b.run()
            tb = np.concatenate([b.trace_by_index(t) for t in range(len(prob_b.trace_list()))], axis=1)
        assert np.array_equal(ta, tb), r.kind
    assert len(seen) >= 3
    model, arrays, _ = S.setup_request(stream[0])
    sdt = K.build_from_arrays(model, arrays).stable_dt
    model.dt = 2.0 * sdt
    with pytest.raises(N.InsemError) as e:
        K.build_solver_from_arrays(model, arrays)
    assert e.value.code == N.ERR_INVALID and "stability limit" in str(e.value)


def _poison(solver):
    """Initial state with one NaN (host-side fault injection through set_state)."""
    medium = solver.media[0]
    u, v, _ = solver.state(medium)
    u = np.array(u, copy=True)
    u[0, u.shape[1] // 2] = np.nan
    solver.set_state(medium, u, v)


def test_nonfinite_request_is_evicted_and_the_mix_is_unaffected(pkg):
    """One request of a running mix goes non-finite (a NaN in its initial
    state): it is marked failed and evicted, and every other request's traces
    still equal its solo run, bit for bit."""
    from insem_b200 import serving as S

    stream = _small_stream()[:6]
    target = stream[2]
    target.init = _poison
    recs = S.Server(chunk_steps=7).run(stream)
    bad = recs[target.rid]
    assert bad.status == "failed" and "NaN" in bad.error, (bad.status, bad.error)
    summ = S.summarize(recs)
    assert summ["completed"] == len(stream) - 1 and summ["failed"] == 1
    for r in stream:
        if r is target:
            continue
        rec = recs[r.rid]
        assert rec.status == "done"
        assert np.array_equal(rec.traces, _solo_traces(r)), (r.rid, r.kind)


def test_plain_server_isolates_a_nonfinite_request(pkg):
    from insem_b200 import serving as S

    stream = _small_stream()[:3]
    stream[1].init = _poison
    recs = S.serve_plain(stream, keep_traces=True)
    assert recs[stream[1].rid].status == "failed"
    for r in (stream[0], stream[2]):
        assert recs[r.rid].status == "done" and np.array_equal(recs[r.rid].traces, _solo_traces(r))
