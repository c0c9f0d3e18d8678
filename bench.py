"""Benchmark of insem's per-time-step path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--nx 1024]

Workload (default): the large coupled Cartesian model -- 1024 x 1024 order-5
elements over 400 m x 400 m, 60 m of water over 8 curved elastic layers,
~26.2M unique GLL points -- built by the native setup from seeded synthetic
parameters (there is no dataset; shapes and value ranges as the benchmark
configuration states them).  A "step" is one central-difference time step of
the whole model.  Metric: GLL-point-updates/s = unique global points summed
over domains x steps / seconds.

value      device time (CUDA events on the solver's stream) of K steps with
           every input resident in HBM; the step touches ~2 GB, larger than
           L2, so no flush is needed.
e2e        the same metric through the C ABI's streamed advance: every step
           copies its source amplitudes in from pinned host memory and its
           receiver sample row (512 receivers) back, wall clock.
roofline   HBM roofline of the whole step: algorithmic bytes per step (the
           fixed B_step formula, ProblemData.algorithmic_bytes_per_step) over
           the step time, against the measured copy bandwidth.
cpu_baseline  the reference's own CPU/OpenMP time loop (oracle build) on the
           same model at 1/16 of the elements (256 x 256), all host cores.

With --gpus N > 1 (torchrun) every rank runs an independent replica (the
path has no exchange step); value = N x per-replica points x steps / the
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


def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value: float, device: int) -> float:
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{device}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device: int):
    import torch

    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize(device)


def cpu_baseline(warmup: int, steps: int) -> dict:
    """The reference's CPU loop on the 1/16 sample (or the oracle port if the reference build is absent)."""
    import __graft_entry__ as entry

    entry.load_package()
    from insem_b200 import cases as K

    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    model = K.config3(nx=REF_SAMPLE_NX, n_receivers=128)
    sys.path.insert(0, str(REPO))
    from oracle import refbench

    if refbench.available():
        r = refbench.run(model, 0.0, warmup, steps)
        return {"value": r["points"] * steps / r["seconds"], "unit": METRIC, "cores": cores, "kind": "reference",
                "sample": f"config3 at nx={REF_SAMPLE_NX} ({r['elements']} elements, {int(r['points'])} points), "
                          f"{steps} steps after {warmup}; setup {r['setup_seconds']:.1f} s excluded",
                "seconds": r["seconds"]}
    import oracle

    prob = K.build(model, stable_dt=None)
    prob.n_steps = warmup + steps
    s = oracle.OracleSolver(prob)
    s.advance(warmup)
    t0 = time.perf_counter()
    s.advance(steps)
    sec = time.perf_counter() - t0
    return {"value": prob.n_global_total() * steps / sec, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"config3 at nx={REF_SAMPLE_NX}, {steps} steps (oracle port, 1 thread)", "seconds": sec}


def run_reference(args, world, rank):
    if rank != 0:
        return
    base = cpu_baseline(args.warmup, args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * base["seconds"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)",
            "config": {"workload": f"config3 coupled 2D Cartesian, order 5, sample nx={REF_SAMPLE_NX}",
                       "l2": "inputs larger than L2"},
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": base["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local, pg):
    import torch

    import __graft_entry__ as entry

    pkg = entry.load_package()
    from insem_b200 import cases as K

    device = local
    torch.cuda.set_device(device)
    total_steps = args.warmup + 2 * args.steps + 2
    model = K.config3(nx=args.nx, n_steps=total_steps)
    t0 = time.perf_counter()
    prob = K.build(model, device=device, stable_dt=args.stable_dt)
    setup_s = time.perf_counter() - t0
    solver = pkg.Solver(prob, device=device, use_graphs=not args.no_graphs)
    solver.advance(args.warmup)
    kps = solver.kernels_per_step if not args.no_graphs else None

    barrier(pg, device)
    with ClockSampler(device) as clocks:
        solver.advance(args.steps)
        barrier(pg, device)
    ms = reduce_max(pg, solver.last_advance_ms, device)
    points = prob.n_global_total()
    value = world * points * args.steps / (ms * 1e-3)

    # e2e: per-step amplitudes in from pinned memory, sample rows out, wall clock
    from insem_b200.stf import amplitudes

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": world * prob.n_global_total() * args.steps / (ms * 1e-3),
                              "ms_per_step": ms / args.steps, "note": "profiling run (no e2e, no baseline)"}))
        solver.close()
        return

    s0 = solver.step
    amp = torch.empty((args.steps, len(prob.sources)), dtype=torch.float32).pin_memory()
    amp.numpy()[:] = amplitudes(prob, s0 + 1, args.steps)
    rows = torch.empty((args.steps + 1, max(solver.n_columns, 1)), dtype=torch.float64).pin_memory()
    barrier(pg, device)
    t0 = time.perf_counter()
    n_rows = solver.advance_streamed(args.steps, amp.numpy(), rows.numpy())
    wall = time.perf_counter() - t0
    wall = reduce_max(pg, wall, device)
    e2e = world * points * args.steps / wall

    hbm, how = peaks()
    b_step = prob.algorithmic_bytes_per_step()
    achieved = b_step / (ms * 1e-3 / args.steps) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded model parameters)",
        "config": {"workload": f"config3 coupled 2D Cartesian {args.nx}x{args.nx} order 5 (water over 8 curved "
                               f"elastic layers)", "points": points, "elements": prob.n_elements_total(),
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (~2 GB touched per step)", "setup_seconds": round(setup_s, 1)},
        "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": 4 * len(prob.sources),
                "d2h_bytes_per_step": 8 * solver.n_columns, "rows": n_rows},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "kernel": "whole step (all kernels of one step)",
                     "algorithmic_bytes_per_step": b_step, "peak_source": how},
        "gpu_launches": (kps or 0) * args.steps,
        "kernels_per_step": kps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and not args.no_cpu:
        try:
            line["cpu_baseline"] = {k: v for k, v in cpu_baseline(1, args.cpu_steps).items() if k != "seconds"}
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": METRIC, "cores": 0, "kind": "unavailable",
                                    "sample": str(exc)[:200]}
    solver.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=1024)
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the streamed end-to-end run")
    ap.add_argument("--no-graphs", action="store_true", help="plain launches instead of the step graph")
    ap.add_argument("--stable-dt", type=float, default=None,
                    help="use this stable time step instead of the device power iteration (profiling runs)")
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
