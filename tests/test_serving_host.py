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
