"""Host side of the serving workload (CPU): the request stream and its models."""

from __future__ import annotations

import numpy as np


def test_stream_is_seeded_and_mixed(pkg):
    from insem_b200 import serving as S

    a = S.request_stream(rate=50.0, window=20.0)
    b = S.request_stream(rate=50.0, window=20.0)
    assert [(r.arrival, r.kind, r.spec) for r in a] == [(r.arrival, r.kind, r.spec) for r in b]
    assert 800 < len(a) < 1200  # Poisson with mean 1000
    kinds = np.array([r.kind for r in a]).astype(str)
    frac_cart = np.mean(np.char.startswith(kinds, "cartesian"))
    frac_m1 = np.mean(kinds == "borehole-m1")
    assert abs(frac_cart - 0.40) < 0.06 and abs(frac_m1 - 0.25) < 0.06
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 1 / 50.0) < 0.003
    for r in a:
        if r.kind.startswith("cartesian"):
            assert 2000 <= r.spec["elements"] <= 200000 and 3 <= r.spec["order"] <= 8
        assert 2e-3 <= r.spec["duration"] <= 8e-3


def test_request_models_set_up(pkg):
    from insem_b200 import serving as S

    stream = S.request_stream(rate=50.0, window=2.0, time_scale=0.01)
    seen = set()
    for r in stream:
        if r.kind in seen:
            continue
        if r.kind.startswith("cartesian"):
            r.spec["elements"] = 3000.0  # small enough for a CPU test
        model, arrays, ne = S.setup_request(r)
        assert ne > 0 and model.duration == r.spec["duration"]
        seen.add(r.kind)
    assert seen == set(S.KINDS)


def test_shipped_tile_table_registers(pkg):
    """The B200 tile table the servers load covers the borehole classes and
    registers every entry (tile sizes change speed only, never results)."""
    import json

    from insem_b200 import autotune, native as N, serving as S

    rows = json.loads(S.DEFAULT_TILE_TABLE.read_text())["tiles"]
    keys = {tuple(r["class"]) for r in rows}
    assert {(ng, N.AXISYM, N.ELASTIC, m, 3 if m else 2) for ng in (5, 6, 7) for m in (0, 1)} <= keys
    before = {k: autotune.current(k) for k in keys}
    try:
        S._load_tiles(S.DEFAULT_TILE_TABLE)
        for r in rows:
            assert autotune.current(tuple(r["class"])) == min(r["te"], autotune.te_max(r["class"][0]))
    finally:
        for k, te in before.items():
            autotune.register(k, te)


def test_pipeline_isolates_failing_and_oversize_requests(pkg, monkeypatch):
    """Host-side failures stay with their request: a request whose setup fails
    (its source lies outside the model) is marked failed with the setup error,
    a request larger than the whole HBM budget is rejected instead of being
    admitted into an empty GPU, and every other request goes through.  The
    device stage is replaced by a stand-in, so this runs without a GPU."""
    import time

    from insem_b200 import serving as S

    stream = S.request_stream(rate=300.0, window=1.0, time_scale=0.004, max_requests=6)
    for r in stream:
        if r.kind.startswith("cartesian"):
            r.spec["elements"] = 2000.0
    bad, big = stream[1].rid, stream[3].rid
    real_model, real_host = S.request_model, S._stage_host

    def model_with_a_stray_source(req):
        m = real_model(req)
        if req.rid == bad:
            m.sources[0].x, m.sources[0].z = 1.0e6, 1.0e6
        return m

    def host_stage(req):
        model, arrays, ne, need = real_host(req)
        return model, arrays, ne, need * 1000 if req.rid == big else need

    class Done:
        n_steps = 1

        @staticmethod
        def n_global_total():
            return 1

    monkeypatch.setattr(S, "request_model", model_with_a_stray_source)
    monkeypatch.setattr(S, "_stage_host", host_stage)
    monkeypatch.setattr(S, "_stage_device", lambda *a, **k: (Done(), object()))
    needs = [real_host(r)[3] for r in stream if r.rid not in (bad, big)]
    recs = {r.rid: S.Record(r.rid, r.kind, r.arrival) for r in stream}
    pipe = S._Pipeline(stream, recs, 0, 10 * max(needs), 2, True, False)
    served = []
    t_end = time.time() + 60.0
    try:
        while pipe.pending() and time.time() < t_end:
            for rid, _, _, need in pipe.poll(0):
                served.append(rid)
                pipe.release(need)
            pipe.idle_wait()
    finally:
        pipe.close()
    assert recs[bad].status == "failed" and "not inside" in recs[bad].error
    assert recs[big].status == "rejected" and "budget" in recs[big].error
    assert sorted(served) == sorted(r.rid for r in stream if r.rid not in (bad, big))
    assert pipe.used == 0
