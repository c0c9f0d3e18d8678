"""Serving: continuous batching of solves that arrive over time.

Requests arrive as a Poisson stream. Each one goes through these stages:
1. Host setup: the native builder runs in worker threads.
2. Admission: the request waits until its device footprint fits the HBM
   budget. Admission is FIFO, and one running ``Batch`` takes every admitted
   request.
3. Batched stepping: the batch advances in short chunks of batched steps.
   Between chunks, newly set-up requests join and completed ones leave.
4. Streaming: every step streams all active requests' sample rows back to
   the host, so a request's traces are on the host when its last step ends.
   Each request's fields, sources (their time-function tables) and receivers
   stay resident on the device.

Latency is measured two ways:
- from admission to the last trace sample on the host;
- from arrival, which adds host setup and queueing.

The same stream can be served by the plain path instead: one solve at a
time, each with its own step graphs, in arrival order.

Batching does not change results: each request's traces and fields are those
it gets alone, bit for bit (tests/test_gpu_serving.py).

Failures stay with the request that caused them.  A request whose setup
fails (a source outside its medium, an unknown material region, ...), whose
device set-up fails, or whose footprint exceeds the whole HBM budget is
marked failed or rejected, with the error, and the stream goes on.  A batch
member whose fields turn non-finite is found when its last step runs, marked
failed and evicted; the members stepping beside it are unaffected (their
arrays are their own) and complete normally.

The reference has no serving loop. Its hook for one is one ``Simulation``
per thread (python/src/bindings.cpp:336-337).
"""

from __future__ import annotations

import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path
from dataclasses import dataclass
from typing import Callable, Dict, List, Optional

import numpy as np

from . import cases as K
from . import native as N
from .batch import Batch
from .problem import ProblemData
from .solver import Solver

KINDS = ("cartesian-acoustic", "cartesian-elastic", "borehole-m0", "borehole-m1")


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the stream starts
    kind: str
    spec: dict
    # Optional initial state: called with the new solver before its first
    # step (for Solver.set_state, as with the reference's set_state).
    init: Optional[Callable] = None


@dataclass
class Record:
    rid: int
    kind: str
    arrival: float
    setup_done: float = float("nan")
    admitted: float = float("nan")
    completed: float = float("nan")
    points: int = 0
    steps: int = 0
    elements: int = 0
    device_bytes: int = 0
    traces: Optional[np.ndarray] = None  # [n_samples][columns], streamed
    status: str = "pending"  # "done", "failed" (error says why) or "rejected" (over the HBM budget)
    error: str = ""


# ---------------------------------------------------------------- workload
def request_stream(rate: float = 50.0, window: float = 20.0, seed: int = 5, time_scale: float = 1.0,
                   max_requests: Optional[int] = None) -> List[Request]:
    """The serving mix as a Poisson stream (`rate` per second over `window` s):
    - 40 % Cartesian 2D, acoustic or elastic, 2k-200k elements, order 3-8;
    - 35 % axisymmetric monopole boreholes;
    - 25 % axisymmetric dipole boreholes.
    The boreholes are drawn from the batched workload's models, with their
    calibrated geometry. Simulated durations are U(2, 8) ms x `time_scale`."""
    rng = np.random.default_rng(seed)
    c4 = K.config4_params(256, 4)
    by_m = {0: [p for p in c4 if p["m"] == 0], 1: [p for p in c4 if p["m"] == 1]}
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > window or (max_requests is not None and len(out) >= max_requests):
            break
        u = rng.random()
        duration = float(rng.uniform(2e-3, 8e-3)) * time_scale
        if u < 0.40:
            elastic = bool(rng.random() < 0.5)
            spec = dict(elements=float(np.exp(rng.uniform(np.log(2000.0), np.log(200000.0)))),
                        order=int(rng.integers(3, 9)), duration=duration,
                        vp=float(rng.uniform(1400.0, 1600.0)) if not elastic else float(rng.uniform(2000.0, 5000.0)),
                        vs_ratio=float(rng.uniform(0.45, 0.6)), rho=float(rng.uniform(1000.0, 2700.0)))
            out.append(Request(len(out), t, "cartesian-elastic" if elastic else "cartesian-acoustic", spec))
        else:
            m = 0 if u < 0.75 else 1
            p = by_m[m][int(rng.integers(0, len(by_m[m])))]
            out.append(Request(len(out), t, f"borehole-m{m}", dict(c4=p["index"], duration=duration)))
    return out


def request_model(req: Request) -> K.Model:
    s = req.spec
    if req.kind.startswith("borehole"):
        p = K.config4_params(256, 4)[s["c4"]]
        geo = K.config4_geometry_table(256, 4)
        return K.config4_model(p, *(geo[s["c4"]] if geo else (6.0, 4.0)), duration=s["duration"])
    # Cartesian: nx x nz elements of 0.05 m; Stacey on the sides and bottom, free top
    n = s["elements"]
    nx = max(8, int(round(np.sqrt(n))))
    nz = max(8, int(round(n / nx)))
    h = 0.05
    w, d = nx * h, nz * h
    f0 = 8000.0
    bcs = {K.BOTTOM: "absorbing", K.LEFT: "absorbing", K.RIGHT: "absorbing", K.TOP: "free"}
    if req.kind == "cartesian-acoustic":
        m = K.rectangle((0.0, w), (-d, 0.0), nx=nx, nz=nz)
        mats = {0: K.Material.acoustic(s["vp"], 1000.0)}
        src = K.Source("monopole", 0.5 * w, -0.5 * d, stf=K.ricker(f0))
        recs = [K.Receiver(f"r{i}", (0.2 + 0.15 * i) * w, -0.25 * d, ["pressure"]) for i in range(5)]
    else:
        vp = s["vp"]
        m = K.rectangle((0.0, w), (-d, 0.0), nx=nx, nz=nz, material=1)
        mats = {1: K.Material.elastic(vp, vp * s["vs_ratio"], s["rho"])}
        src = K.Source("force", 0.5 * w, -0.5 * d, (0.0, 1.0, 0.0), K.ricker(f0))
        recs = [K.Receiver(f"r{i}", (0.2 + 0.15 * i) * w, -0.1 * d, ["velocity"]) for i in range(5)]
    return K.Model(m, order=s["order"], materials=mats, boundaries=bcs, sources=[src], receivers=recs,
                   duration=s["duration"])


def setup_request(req: Request):
    """Host setup of a request (worker thread): (model, arrays, elements)."""
    model = request_model(req)
    arrays = K.setup_arrays(model)
    return model, arrays, K.n_elements(arrays)


def device_bytes_estimate(prob: ProblemData) -> int:
    """Device footprint of a solve on the tiled path:
    - element data and numbering, kept twice (the two-pass path's copy and
      the tiled layout);
    - the five field arrays;
    - a margin for traces and small tables."""
    host = 0

    def walk(x):
        nonlocal host
        if isinstance(x, np.ndarray):
            host += x.nbytes
        elif isinstance(x, (list, tuple)):
            for y in x:
                walk(y)
        elif hasattr(x, "__dict__"):
            for y in vars(x).values():
                walk(y)

    walk(prob.domains)
    fields = sum(20 * d.ncomp * d.n_global for d in prob.domains)
    return int(2 * host + fields + (4 << 20))


def mem_info(device: int):
    """(free, total) device memory in bytes."""
    import ctypes as C

    f, t = C.c_int64(), C.c_int64()
    N.check(N.lib().insem_cuda_mem_info(device, C.byref(f), C.byref(t)))
    return f.value, t.value


def _stage_host(req: Request):
    """Stage A (host, worker thread): model, native setup, footprint estimate."""
    model, arrays, ne = setup_request(req)
    probe = dict(arrays)
    probe.update({"problem.dt": np.asarray(1.0), "problem.n_steps": np.asarray(0),
                  "problem.stable_dt": np.asarray(0.0)})
    return model, arrays, ne, device_bytes_estimate(ProblemData.from_npz(probe))


def _stage_device(model, arrays, device: int, use_graphs: bool, prepare: bool, init=None):
    """Stage B (device, worker thread): dt from the power iteration, the solver,
    the request's initial state (and, for the batched server, its initial step
    and predictor)."""
    prob, s = K.build_solver_from_arrays(model, arrays, device=device, use_graphs=use_graphs)
    try:
        if init is not None:
            init(s)
        if prepare:
            s.prepare_for_batch()
    except Exception:
        s.close()
        raise
    return prob, s


class _Pipeline:
    """Arrivals -> host setup -> FIFO admission by HBM budget -> device setup.
    Solvers come out in arrival order, ready to step."""

    def __init__(self, stream: List[Request], recs: Dict[int, Record], device: int, budget: int, workers: int,
                 use_graphs: bool, prepare: bool):
        self.stream, self.recs, self.device, self.budget = stream, recs, device, budget
        self.use_graphs = use_graphs
        self.prepare = prepare
        self.pool = ThreadPoolExecutor(max_workers=workers)
        self.host: Dict[int, object] = {}     # rid -> future of stage A
        self.waiting: deque = deque()        # (rid, model, arrays, bytes), arrival order
        self.dev: deque = deque()            # (rid, bytes, future of stage B), admission order
        self.used = 0
        self.i = 0
        self.stream_by_rid = {r.rid: r for r in stream}
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def pending(self) -> bool:
        return self.i < len(self.stream) or bool(self.host) or bool(self.waiting) or bool(self.dev)

    def fail(self, rid: int, error: Exception, status: str = "failed") -> None:
        rec = self.recs[rid]
        rec.status, rec.error, rec.completed = status, f"{type(error).__name__}: {error}", float("nan")

    def poll(self, running: int) -> List[tuple]:
        """Advances the pipeline; returns (rid, problem, solver, bytes) now ready.
        Requests whose setup fails, or that could never fit the budget, leave
        the pipeline marked failed or rejected."""
        now = self.now()
        while self.i < len(self.stream) and self.stream[self.i].arrival <= now:
            r = self.stream[self.i]
            self.host[r.rid] = self.pool.submit(_stage_host, r)
            self.i += 1
        for rid in sorted(self.host):
            f = self.host[rid]
            if not f.done():
                break  # keep arrival order
            del self.host[rid]
            try:
                model, arrays, ne, need = f.result()
            except Exception as e:  # the request's own setup failed
                self.fail(rid, e)
                continue
            rec = self.recs[rid]
            rec.setup_done, rec.elements, rec.device_bytes = self.now(), ne, need
            if need > self.budget:
                self.fail(rid, MemoryError(f"needs {need} bytes of device memory, the budget is {self.budget}"),
                          "rejected")
                continue
            self.waiting.append((rid, model, arrays, need))
        while self.waiting:
            rid, model, arrays, need = self.waiting[0]
            if (running or self.dev) and self.used + need > self.budget:
                break  # FIFO admission: wait for completions to free memory
            self.waiting.popleft()
            self.used += need
            self.recs[rid].admitted = self.now()
            self.dev.append((rid, need, self.pool.submit(_stage_device, model, arrays, self.device,
                                                         self.use_graphs, self.prepare,
                                                         self.stream_by_rid[rid].init)))
        out = []
        while self.dev and self.dev[0][2].done():
            rid, need, f = self.dev.popleft()
            try:
                prob, solver = f.result()
            except Exception as e:  # device set-up of this request failed
                self.release(need)
                self.fail(rid, e)
                continue
            rec = self.recs[rid]
            rec.points, rec.steps = prob.n_global_total(), prob.n_steps
            out.append((rid, prob, solver, need))
        return out

    def release(self, need: int) -> None:
        self.used -= need

    def idle_wait(self) -> None:
        if self.i < len(self.stream) and not self.host and not self.waiting and not self.dev:
            time.sleep(max(0.0, min(0.002, self.stream[self.i].arrival - self.now())))
        else:
            time.sleep(0.0005)

    def close(self) -> None:
        self.pool.shutdown(wait=True)


# ------------------------------------------------------------------ servers
# Tile sizes that autotune.tune_batched measured on a B200 for the borehole
# tile classes (axisymmetric elastic, ngll 5-7, m = 0 and 1: the classes of
# every borehole request), in autotune.save's format.  Other classes keep the
# occupancy-based default.  Tile sizes change speed only, never results.
DEFAULT_TILE_TABLE = Path(__file__).resolve().parent / "data" / "tile_table_b200.json"


def _load_tiles(tile_table) -> None:
    """Registers a saved tile table for the whole process (None: keep the current choices)."""
    if tile_table:
        from . import autotune

        autotune.load(str(tile_table))


class Server:
    """Continuous-batching server over one Batch on one device."""

    def __init__(self, device: int = 0, hbm_budget: Optional[int] = None, chunk_steps: int = 64,
                 workers: Optional[int] = None, use_graphs: bool = True, tile_table=DEFAULT_TILE_TABLE):
        import os

        _load_tiles(tile_table)
        self.device = device
        free, _ = mem_info(device)
        self.budget = int(hbm_budget) if hbm_budget else int(0.8 * free)
        self.chunk = chunk_steps
        self.workers = workers or max(1, min(32, os.cpu_count() or 1))
        self.use_graphs = use_graphs

    def run(self, stream: List[Request], keep_traces: bool = True) -> Dict[int, Record]:
        recs = {r.rid: Record(r.rid, r.kind, r.arrival) for r in stream}
        batch = Batch(device=self.device, use_graphs=self.use_graphs)
        pipe = _Pipeline(stream, recs, self.device, self.budget, self.workers, self.use_graphs, True)
        members: Dict[int, tuple] = {}    # batch index -> (rid, member, bytes, streamed row blocks)
        try:
            while pipe.pending() or members:
                for rid, prob, solver, need in pipe.poll(len(members)):
                    m = batch.adopt(solver)
                    members[m.index] = (rid, m, need, [])
                if not members:
                    pipe.idle_wait()
                    continue
                # a full chunk: members that finish inside it idle on the device
                act = batch.active_members()
                left = {m.index: m.n_steps - m.step for m in act}
                _, row_cols = batch.stream_layout()
                rows = np.empty((self.chunk, max(row_cols, 1)))
                try:
                    done = batch.advance_streamed(self.chunk, None, rows)
                except N.InsemError as e:
                    if e.code != N.ERR_NONFINITE:
                        raise
                    # the steps ran and the rows are in; the members that
                    # failed are marked and leave below
                    done = min(self.chunk, max(left.values()))
                col = 0
                for m in act:
                    nc = m.n_columns
                    if keep_traces:
                        members[m.index][3].append(rows[:min(done, left[m.index]), col:col + nc].copy())
                    col += nc
                for idx in [j for j, (_, m, _, _) in members.items() if m.step >= m.n_steps]:
                    rid, m, need, blocks = members.pop(idx)
                    r = recs[rid]
                    if m.failed:
                        pipe.fail(rid, N.InsemError(N.ERR_NONFINITE, "the solution contains NaN or Inf"))
                        batch.remove(m)
                        pipe.release(need)
                        continue
                    r.completed, r.status = pipe.now(), "done"
                    if keep_traces:
                        n_tr = len(m.problem.trace_list())
                        first = (np.concatenate([m.trace_by_index(t)[:1] for t in range(n_tr)], axis=1)
                                 if n_tr else np.zeros((1, 0)))
                        r.traces = np.concatenate([first] + blocks, axis=0)
                    batch.remove(m)
                    pipe.release(need)
        finally:
            pipe.close()
            batch.close()
        return recs


def serve_plain(stream: List[Request], device: int = 0, workers: Optional[int] = None,
                keep_traces: bool = False, hbm_budget: Optional[int] = None,
                tile_table=DEFAULT_TILE_TABLE) -> Dict[int, Record]:
    """The plain path on the same stream, the same setup pipeline and the same
    tile sizes. Requests are solved one at a time in arrival order, each with
    its own step graphs."""
    import os

    _load_tiles(tile_table)
    recs = {r.rid: Record(r.rid, r.kind, r.arrival) for r in stream}
    free, _ = mem_info(device)
    pipe = _Pipeline(stream, recs, device, int(hbm_budget) if hbm_budget else int(0.8 * free),
                     workers or max(1, min(32, os.cpu_count() or 1)), True, False)
    ready: deque = deque()
    try:
        while pipe.pending() or ready:
            ready.extend(pipe.poll(1 if ready else 0))
            if not ready:
                pipe.idle_wait()
                continue
            rid, prob, s, need = ready.popleft()
            with s:
                try:
                    s.run()
                except N.InsemError as e:
                    if e.code != N.ERR_NONFINITE:
                        raise
                    pipe.fail(rid, e)
                    pipe.release(need)
                    continue
                if keep_traces:
                    n_tr = len(prob.trace_list())
                    recs[rid].traces = (np.concatenate([s.trace_by_index(t) for t in range(n_tr)], axis=1)
                                        if n_tr else np.zeros((prob.n_steps + 1, 0)))
            recs[rid].completed, recs[rid].status = pipe.now(), "done"
            pipe.release(need)
    finally:
        pipe.close()
    return recs


def summarize(recs: Dict[int, Record]) -> dict:
    """p50/p99 latency (from admission and from arrival) and aggregate throughput."""
    done = [r for r in recs.values() if r.status == "done"]
    failed = sum(r.status == "failed" for r in recs.values())
    rejected = sum(r.status == "rejected" for r in recs.values())
    if not done:
        return {"completed": 0, "requests": len(recs), "failed": failed, "rejected": rejected}
    lat_adm = np.array([r.completed - r.admitted for r in done])
    lat_arr = np.array([r.completed - r.arrival for r in done])
    span = max(r.completed for r in done) - min(r.arrival for r in done)
    updates = sum(r.points * r.steps for r in done)
    return {"completed": len(done), "requests": len(recs), "failed": failed, "rejected": rejected,
            "p50_ms_from_admission": 1e3 * float(np.percentile(lat_adm, 50)),
            "p99_ms_from_admission": 1e3 * float(np.percentile(lat_adm, 99)),
            "p50_ms_from_arrival": 1e3 * float(np.percentile(lat_arr, 50)),
            "p99_ms_from_arrival": 1e3 * float(np.percentile(lat_arr, 99)),
            "seconds": span, "point_updates": int(updates), "value": updates / span if span > 0 else None,
            "elements_mean": float(np.mean([r.elements for r in done])),
            "steps_mean": float(np.mean([r.steps for r in done]))}
