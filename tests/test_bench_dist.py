"""bench.py's multi-process logic on CPU (gloo, world size 2): the replicas
share no data, so a run's only collectives are the barrier and the max of the
ranks' device times; the whole-job value counts every replica's work over
the slowest rank's time."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import sys

    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(REPO))
    import bench

    w, r, local, pg = bench.dist_setup(world, backend="gloo")
    try:
        assert (w, r, local) == (world, rank, rank)
        bench.barrier(pg, None)
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
        mx = bench.reduce_max(pg, ms, None)
        out.put((rank, mx, bench.replica_value(w, 1000, mx)))
        bench.barrier(pg, None)
    finally:
        pg.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, mx, value in res:
        assert mx == 15.0
        assert value == pytest.approx(2 * 1000 / 15e-3)


def test_single_process_has_no_group(monkeypatch):
    import sys

    sys.path.insert(0, str(REPO))
    import bench

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    w, r, local, pg = bench.dist_setup(1)
    assert (w, r, local, pg) == (1, 0, 0, None)
    assert bench.reduce_max(None, 3.5, None) == 3.5
