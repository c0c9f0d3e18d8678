"""Benchmark of insem's per-time-step path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|config3] [--models 256] [--nx 1024]

Metric: GLL-point-updates/s = unique global points summed over domains and
solves x steps / seconds (setup and the stable-dt power iteration excluded).

Default workload (batched): 256 independent axisymmetric borehole models
(seeded: hole radius, monopole / dipole half each, 1-6 beds incl. slow
formations, casing in 30 %, GLL order 4-6, 5k-80k elements after AMR, 13
receivers, 5 ms), built by the native setup.  A step is one batched step:
one time step of every model (each with its own dt).

value      device time (CUDA events) of K batched steps, every input resident
           in HBM; a batched step touches ~16 GB, far more than L2.
plain      the same models with the plain one-solve-per-launch path (each
           solve's own step graph, solves one after another), device time.
e2e        the same metric through the C ABI's streamed batched steps: every
           step copies all models' source amplitudes in from pinned host
           memory and all models' sample rows back, wall clock.
roofline   HBM roofline of the tile kernels (the dominant launches): their
           algorithmic bytes per batched step (element terms + points finished
           in tiles, the fixed B_step formula split by point class) over their
           CUDA-event time per step, measured on plain launches after the
           timed region; step_roofline: the whole step's B_step over the
           timed step time.
plain_config3  the large coupled Cartesian model (1024 x 1024 order-5
           elements, ~26.2M points) on the plain path: value and roofline.
cpu_baseline  the reference's own CPU/OpenMP time loop (oracle build) on a
           sample of the same models, all host cores.

With --gpus N > 1 (torchrun) every rank runs an independent replica (the
path has no exchange step); value = sum over ranks of point-updates / the
slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "GLL-point-updates/s"
FALLBACK_HBM_GBS = 6650.0
REF_SAMPLE_NX = 256


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def traffic(name: str, algorithmic_bytes: int):
    """DRAM bytes (read + write) of the roofline's kernels, from the ncu capture
    recorded in data/dram_traffic_b200.json for this workload: the captured
    DRAM bytes per algorithmic byte, times this run's algorithmic bytes (the
    capture is a smaller case of the same kernels; DRAM bytes grow with the
    elements and points processed)."""
    p = REPO / "in-house-sem_b200" / "data" / "dram_traffic_b200.json"
    if not p.exists():
        return None, None
    rec = json.loads(p.read_text()).get(name)
    if not rec:
        return None, None
    return rec["dram_per_algorithmic_byte"] * algorithmic_bytes, rec["source"]


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "100"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self._proc:
            time.sleep(0.25)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup(n_gpus: int, backend: str = "nccl"):
    """Rank, world and process group from the torchrun environment (replicas:
    no collective touches the data path; the group carries the barrier and
    the max over ranks only).  backend "gloo" runs the same logic on CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value: float, device) -> float:
    """Max of `value` over ranks (device None: a CPU tensor, for gloo)."""
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cpu" if device is None else f"cuda:{device}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    import torch

    if pg is not None:
        pg.barrier()
    if device is not None:
        torch.cuda.synchronize(device)


def replica_value(world: int, updates_per_rank: int, max_ms: float) -> float:
    """Whole-job GLL-point-updates/s of N replicas: every rank did the same
    work; the slowest rank's device time bounds the job."""
    return world * updates_per_rank / (max_ms * 1e-3)


def _cpu_env():
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    return cores


def cpu_baseline_config3(warmup: int, steps: int) -> dict:
    """The reference's CPU loop on config3 at 1/16 of the elements (or the oracle port without the reference build)."""
    import __graft_entry__ as entry

    entry.load_package()
    from insem_b200 import cases as K

    cores = _cpu_env()
    model = K.config3(nx=REF_SAMPLE_NX, n_receivers=128)
    from oracle import refbench

    if refbench.available():
        r = refbench.run(model, 0.0, warmup, steps)
        return {"value": r["points"] * steps / r["seconds"], "unit": METRIC, "cores": cores, "kind": "reference",
                "sample": f"config3 at nx={REF_SAMPLE_NX} ({r['elements']} elements, {int(r['points'])} points), "
                          f"{steps} steps after {warmup}; setup {r['setup_seconds']:.1f} s excluded",
                "seconds": r["seconds"], "steps": steps}
    import oracle

    prob = K.build(model, stable_dt=None)
    prob.n_steps = warmup + steps
    s = oracle.OracleSolver(prob)
    s.advance(warmup)
    t0 = time.perf_counter()
    s.advance(steps)
    sec = time.perf_counter() - t0
    return {"value": prob.n_global_total() * steps / sec, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"config3 at nx={REF_SAMPLE_NX}, {steps} steps (oracle port, 1 thread)", "seconds": sec,
            "steps": steps}


def cpu_baseline_config4(warmup: int, steps: int, sample_models: int = 4) -> dict:
    """The reference's CPU loop on the first `sample_models` batched borehole
    models in sequence, each on all host cores, at the dt the device uses
    (or the oracle port without the reference build)."""
    import __graft_entry__ as entry

    entry.load_package()
    from insem_b200 import cases as K

    cores = _cpu_env()
    from oracle import refbench

    params = K.config4_params(256, 4)[:sample_models]
    geo = K.config4_geometry_table(256, 4)
    updates, seconds, elems = 0.0, 0.0, 0
    if refbench.available():
        for i, p in enumerate(params):
            model = K.config4_model(p, *(geo[i] if geo else (6.0, 4.0)))
            r = refbench.run(model, 0.0, warmup, steps)
            updates += r["points"] * steps
            seconds += r["seconds"]
            elems += r["elements"]
        return {"value": updates / seconds, "unit": METRIC, "cores": cores, "kind": "reference",
                "sample": f"config4 models 0-{sample_models - 1} ({elems} elements) in sequence, {steps} steps each "
                          f"after {warmup}, reference dt; setup excluded",
                "seconds": seconds, "steps": steps}
    import oracle

    for i, p in enumerate(params):
        model = K.config4_model(p, *(geo[i] if geo else (6.0, 4.0)))
        prob = K.build(model, stable_dt=1e-7)
        prob.n_steps = warmup + steps
        s = oracle.OracleSolver(prob)
        s.advance(warmup)
        t0 = time.perf_counter()
        s.advance(steps)
        seconds += time.perf_counter() - t0
        updates += prob.n_global_total() * steps
    return {"value": updates / seconds, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"config4 models 0-{sample_models - 1}, {steps} steps each (oracle port, 1 thread)",
            "seconds": seconds, "steps": steps}


def run_reference(args, world, rank):
    if rank != 0:
        return
    # exactly --steps timed steps after --warmup, each a bounded sample of the workload
    if args.workload == "config3":
        base = cpu_baseline_config3(args.warmup, args.steps)
        workload = f"config3 coupled 2D Cartesian, order 5, sample nx={REF_SAMPLE_NX}"
    else:
        base = cpu_baseline_config4(args.warmup, args.steps)
        workload = "config4 batched boreholes (reference: models in sequence, all host cores)"
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": base["steps"], "warmup": args.warmup, "ms_per_step": 1e3 * base["seconds"] / base["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded model parameters)",
            "config": {"workload": workload, "l2": "inputs larger than L2"},
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": base["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_config3(args, world, rank, device, pg, headline: bool) -> dict:
    """The large coupled Cartesian model on the plain path."""
    import torch

    import __graft_entry__ as entry

    pkg = entry.load_package()
    from insem_b200 import cases as K
    from insem_b200.stf import amplitudes

    steps = args.steps if headline else args.config3_steps
    total_steps = args.warmup + 2 * steps + 2
    model = K.config3(nx=args.nx, n_steps=total_steps)
    t0 = time.perf_counter()
    prob = K.build(model, device=device, stable_dt=args.stable_dt)
    setup_s = time.perf_counter() - t0
    solver = pkg.Solver(prob, device=device, use_graphs=not args.no_graphs)
    solver.advance(args.warmup)
    kps = solver.kernels_per_step if not args.no_graphs else None
    barrier(pg, device)
    with ClockSampler(device) as clocks:
        solver.advance(steps)
        barrier(pg, device)
    ms = reduce_max(pg, solver.last_advance_ms, device)
    points = prob.n_global_total()
    hbm, how = peaks()
    b_step = prob.algorithmic_bytes_per_step()
    achieved = b_step / (ms * 1e-3 / steps) / 1e9
    dram, dram_src = traffic("config3_step", b_step)
    out = {"value": replica_value(world, points * steps, ms), "ms_per_step": ms / steps, "steps": steps,
           "workload": f"config3 coupled 2D Cartesian {args.nx}x{args.nx} order 5 (water over 8 curved elastic layers)",
           "points": points, "elements": prob.n_elements_total(), "setup_seconds": round(setup_s, 1),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                        "traffic": dram, "traffic_source": dram_src, "kernel": "whole step (all kernels of one step)",
                        "algorithmic_bytes_per_step": b_step, "peak_source": how},
           "kernels_per_step": kps, "clocks": clocks.summary()}
    if headline and not args.no_e2e:
        s0 = solver.step
        amp = torch.empty((steps, len(prob.sources)), dtype=torch.float32).pin_memory()
        amp.numpy()[:] = amplitudes(prob, s0 + 1, steps)
        rows = torch.empty((steps + 1, max(solver.n_columns, 1)), dtype=torch.float64).pin_memory()
        barrier(pg, device)
        t0 = time.perf_counter()
        n_rows = solver.advance_streamed(steps, amp.numpy(), rows.numpy())
        wall = reduce_max(pg, time.perf_counter() - t0, device)
        out["e2e"] = {"value": world * points * steps / wall, "unit": METRIC, "h2d_bytes_per_step": 4 * len(prob.sources),
                      "d2h_bytes_per_step": 8 * solver.n_columns, "rows": n_rows}
    solver.close()
    return out


def build_config4(args, device):
    """The batched borehole models as (params, problem, solver): setups in a
    thread pool, the tile autotuner on the largest model of each tile class,
    then the solvers."""
    import __graft_entry__ as entry

    pkg = entry.load_package()
    from insem_b200 import autotune
    from insem_b200 import cases as K

    from concurrent.futures import ThreadPoolExecutor

    probs, chunk = [], []

    def flush():
        with ThreadPoolExecutor(max_workers=len(chunk)) as ex:
            probs.extend(ex.map(lambda c: (c[0], K.build_from_arrays(c[1], c[2], device=device)), chunk))
        chunk.clear()

    # stable-dt estimates in threads, one chunk of models' host arrays held at a time
    for p, model, arrays, ne, geo in K.config4(args.models, workers=max(1, min(4, args.setup_threads))):
        chunk.append((p, model, arrays))
        if len(chunk) == max(1, args.setup_threads):
            flush()
    if chunk:
        flush()
    t0 = time.perf_counter()
    table = None if args.no_autotune else autotune.tune_batched([q for _, q in probs], device=device)
    tune_s = time.perf_counter() - t0
    if table and args.save_tiles:
        autotune.save(table, args.save_tiles)
    out = [(p, prob, pkg.Solver(prob, device=device, use_graphs=not args.no_graphs)) for p, prob in probs]
    return out, {"classes": autotune.summary(table), "seconds": round(tune_s, 1)} if table else None


def bench_config4(args, world, rank, device, pg) -> dict:
    import torch

    import __graft_entry__ as entry

    pkg = entry.load_package()
    from insem_b200.stf import amplitudes

    t0 = time.perf_counter()
    models, tuned = build_config4(args, device)
    setup_s = time.perf_counter() - t0
    points = sum(prob.n_global_total() for _, prob, _ in models)
    elements = sum(prob.n_elements_total() for _, prob, _ in models)
    b_step = sum(prob.algorithmic_bytes_per_step() for _, prob, _ in models)
    split = [s.algorithmic_bytes_split() for _, _, s in models]
    tile_bytes = sum(t for t, _ in split)

    # plain: every solve alone, its own step graph, one after another
    plain_ms, plain_updates = 0.0, 0
    for _, prob, s in models:
        s.advance(args.warmup)
        s.advance(args.plain_steps)
        plain_ms += s.last_advance_ms
        plain_updates += prob.n_global_total() * args.plain_steps
    plain_ms = reduce_max(pg, plain_ms, device)
    plain_value = replica_value(world, plain_updates, plain_ms)

    # batched
    batch = pkg.Batch(device=device, use_graphs=not args.no_graphs, tile_streams=args.tile_streams)
    members = [batch.adopt(s) for _, _, s in models]
    batch.advance(args.warmup)
    barrier(pg, device)
    with ClockSampler(device) as clocks:
        batch.advance(args.steps)
        barrier(pg, device)
    updates = batch.point_updates
    ms = reduce_max(pg, batch.last_advance_ms, device)
    value = replica_value(world, updates, ms)
    kps = batch.kernels_per_step if not args.no_graphs else None

    line_e2e = None
    if not args.no_e2e:
        k = min(args.steps, batch.steps_to_next_completion)
        act = batch.active_members()
        amp_cols, row_cols = batch.stream_layout()
        amp = torch.empty((k, max(amp_cols, 1)), dtype=torch.float32).pin_memory()
        an = amp.numpy()
        col = 0
        for m in act:
            nsrc = len(m.problem.sources)
            an[:, col:col + nsrc] = amplitudes(m.problem, m.step + 1, k)
            col += nsrc
        rows = torch.empty((k, max(row_cols, 1)), dtype=torch.float64).pin_memory()
        barrier(pg, device)
        t0 = time.perf_counter()
        done = batch.advance_streamed(k, amp, rows)
        wall = reduce_max(pg, time.perf_counter() - t0, device)
        line_e2e = {"value": world * batch.point_updates / wall, "unit": METRIC, "h2d_bytes_per_step": 4 * amp_cols,
                    "d2h_bytes_per_step": 8 * row_cols, "steps": done}

    # dominant launches: the tile kernels, CUDA events around them on plain launches
    tile_ms, step_ms = batch.profile(args.profile_steps)
    hbm, how = peaks()
    per_step_tile_s = tile_ms * 1e-3 / args.profile_steps
    achieved = tile_bytes / per_step_tile_s / 1e9
    step_achieved = b_step / (ms * 1e-3 / args.steps) / 1e9
    dram, dram_src = traffic("batched_tiles", tile_bytes)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded model parameters)",
        "config": {"workload": f"config4: {len(models)} axisymmetric borehole models batched (GLL order 4-6, "
                               f"m=0/1 half each, 5k-80k elements, casing in 30 %)",
                   "models": len(models), "points": points, "elements": elements,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": f"inputs larger than L2 (~{b_step / 1e9:.1f} GB touched per batched step)",
                   "setup_seconds": round(setup_s, 1)},
        "plain": {"value": plain_value, "unit": METRIC, "steps_per_model": args.plain_steps,
                  "ms_total": plain_ms, "path": "one solve per launch: each model's own step graph, in sequence"},
        "batched_over_plain": value / plain_value,
        "e2e": line_e2e,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": dram, "traffic_source": dram_src,
                     "kernel": "tile_batch_kernel (all tile classes of one batched step)",
                     "algorithmic_bytes_per_launch_group": tile_bytes, "ms_per_launch_group": tile_ms / args.profile_steps,
                     "tile_share_of_step": tile_ms / step_ms if step_ms > 0 else None, "peak_source": how},
        "step_roofline": {"achieved": step_achieved, "frac": step_achieved / hbm, "algorithmic_bytes_per_step": b_step},
        "gpu_launches": (kps or 0) * args.steps,
        "kernels_per_step": kps,
        "clocks": clocks.summary(),
        "autotune": tuned,
    }
    batch.close()
    return line


def bench_serving(args, device) -> dict:
    """The serving stream through the continuous-batching server and through
    the plain path (one solve at a time), on the same requests, at each
    arrival rate of --serve-rates (rates one GPU sustains, so latency is
    service time plus short queueing) and at --serve-rate (the stated 50/s,
    above one GPU's capacity: latency there is mostly queueing)."""
    import __graft_entry__ as entry

    entry.load_package()
    from insem_b200 import serving as S

    # warm-up: a short stream of the same mix loads the kernels every class uses
    S.Server(device=device, chunk_steps=args.serve_chunk).run(
        S.request_stream(rate=200.0, window=1.0, seed=55, time_scale=1e-3, max_requests=24), keep_traces=False)

    def point(rate: float, window: float, seed: int) -> dict:
        stream = S.request_stream(rate=rate, window=window, seed=seed, time_scale=args.serve_scale)
        t0 = time.perf_counter()
        batched = S.summarize(S.Server(device=device, chunk_steps=args.serve_chunk).run(stream, keep_traces=False))
        wall_b = time.perf_counter() - t0
        t0 = time.perf_counter()
        plain = S.summarize(S.serve_plain(stream, device=device))
        wall_p = time.perf_counter() - t0
        out = {"rate_per_s": rate, "window_s": window, "requests": len(stream), "batched": batched, "plain": plain,
               "wall_seconds": {"batched": round(wall_b, 1), "plain": round(wall_p, 1)}}
        if batched.get("value") and plain.get("value"):
            out["batched_over_plain"] = batched["value"] / plain["value"]
        return out

    rates = [float(x) for x in args.serve_rates.split(",") if x.strip()] if args.serve_rates else []
    points = [point(r, args.serve_window_sustained, 5 + i) for i, r in enumerate(rates)]
    overload = point(args.serve_rate, args.serve_window, 5)
    return {"workload": "Poisson arrivals: 40 % Cartesian (2k-200k elements, order 3-8), 35 % monopole and 25 % "
                        f"dipole boreholes from the batched set; simulated durations U(2, 8) ms x {args.serve_scale:g}; "
                        "the batched and the plain server serve the same requests at each rate",
            "sustained": points, "overload": overload,
            "batched_over_plain": overload.get("batched_over_plain")}


def run_ours(args, world, rank, local, pg):
    import torch

    device = local
    torch.cuda.set_device(device)
    if args.workload == "config3":
        r = bench_config3(args, world, rank, device, pg, headline=True)
        line = {
            "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": world, "steps": r["steps"],
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded model parameters)",
            "config": {"workload": r["workload"], "points": r["points"], "elements": r["elements"],
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (~2 GB touched per step)", "setup_seconds": r["setup_seconds"]},
            "e2e": r.get("e2e"), "roofline": r["roofline"],
            "gpu_launches": (r["kernels_per_step"] or 0) * r["steps"], "kernels_per_step": r["kernels_per_step"],
            "clocks": r["clocks"],
        }
    else:
        line = bench_config4(args, world, rank, device, pg)
        if not args.no_serving:
            line["serving"] = bench_serving(args, device)
        if not args.no_config3:
            r = bench_config3(args, world, rank, device, pg, headline=False)
            line["plain_config3"] = {k: r[k] for k in ("value", "ms_per_step", "steps", "workload", "points",
                                                        "roofline", "clocks")}
            line["gpu_launches"] += (r["kernels_per_step"] or 0) * r["steps"]
    if rank == 0 and not args.no_cpu:
        try:
            if args.workload == "config3":
                base = cpu_baseline_config3(1, args.cpu_steps)
            else:
                base = cpu_baseline_config4(1, args.cpu_steps)
            line["cpu_baseline"] = {k: v for k, v in base.items() if k not in ("seconds", "steps")}
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": METRIC, "cores": 0, "kind": "unavailable",
                                    "sample": str(exc)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batched", "config3"], default="batched")
    ap.add_argument("--models", type=int, default=256, help="batched workload: number of models")
    ap.add_argument("--plain-steps", type=int, default=20, help="batched workload: steps per model on the plain path")
    ap.add_argument("--profile-steps", type=int, default=5, help="steps of the event-timed tile profile")
    ap.add_argument("--nx", type=int, default=1024, help="config3 elements per side")
    ap.add_argument("--config3-steps", type=int, default=200, help="steps of the config3 sub-run")
    ap.add_argument("--no-config3", action="store_true", help="skip the config3 sub-run")
    ap.add_argument("--no-autotune", action="store_true", help="batched workload: keep the default tile sizes")
    ap.add_argument("--tile-streams", type=int, default=0,
                    help="batched workload: streams the tile launches of a step spread over (0 = library default)")
    ap.add_argument("--save-tiles", default=None,
                    help="batched workload: write the tuned tile table (JSON, autotune.load format) here")
    ap.add_argument("--setup-threads", type=int, default=16,
                    help="batched workload: host threads building the models and their stable time steps")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving stream")
    ap.add_argument("--serve-rate", type=float, default=50.0, help="serving: mean arrivals per second")
    ap.add_argument("--serve-window", type=float, default=3.0, help="serving: seconds of arrivals at --serve-rate")
    ap.add_argument("--serve-rates", default="1,2,3",
                    help="serving: arrival rates (per s) one GPU sustains, measured besides --serve-rate")
    ap.add_argument("--serve-window-sustained", type=float, default=8.0,
                    help="serving: seconds of arrivals at each of --serve-rates")
    ap.add_argument("--serve-scale", type=float, default=0.25, help="serving: factor on the simulated durations")
    ap.add_argument("--serve-chunk", type=int, default=64, help="serving: batched steps between admissions")
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the streamed end-to-end run")
    ap.add_argument("--no-graphs", action="store_true", help="plain launches instead of the step graphs")
    ap.add_argument("--stable-dt", type=float, default=None,
                    help="config3: use this stable time step instead of the device power iteration (profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
