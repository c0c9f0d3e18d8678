"""Generates the golden fixtures in tests/golden from the reference itself.

Test infrastructure only.  Needs the reference sources and their oracle build
(``make -C oracle/ref``); run from the repository root:

    python tests/golden/make_golden.py

For every case in ``cases.py`` it builds the model through the reference's
own Python API, reads the arrays the reference solver packs for its time loop
(``_refdump.problem``), computes per-block force vectors, gather, assemble and
internal forces on seeded random inputs, runs the time loop and stores the
receiver traces, energy samples and final fields.  The float build (the parity
target) writes ``<case>.npz``; the double build (the FP64 oracle) writes
``<case>_f64.npz`` with traces and energy only; the strict-FP build is run to
check that it agrees bit for bit with the float build on this machine.

Random inputs are regenerated in the tests from the same seeds
(``numpy.random.default_rng(seed)``), so only outputs are stored.

``--timed`` makes the fixtures of the benchmarked configurations instead
(``timed_cases.py``: config 2 at its stated geometry, config 3 at 64 x 64,
six config 4 boreholes, the Gaussian and sampled source time functions).
Their setup arrays are large, so ``timed_<case>.npz`` stores a SHA-256 digest
of every problem array and of the final fields, next to the reference's dt,
stable dt, step counts, receiver traces and energy samples.  The double build
runs the same model with the float build's dt (so samples align) and writes
``timed_<case>_f64.npz`` with traces and energy.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
REF_BUILD = REPO / "oracle" / "_ref"

# Seeds of the random test inputs (shared with tests/golden_io.py).
SEED_BLOCK = 101
SEED_GATHER = 202
SEED_ASSEMBLE = 303
SEED_FORCES = 404


def flatten(prefix: str, obj, out: dict) -> None:
    """Nested dict/list of arrays -> flat npz keys joined by '.'."""
    if isinstance(obj, dict):
        for k, v in obj.items():
            flatten(f"{prefix}.{k}" if prefix else str(k), v, out)
    elif isinstance(obj, (list, tuple)) and obj and isinstance(obj[0], dict):
        out[f"{prefix}.count"] = np.int64(len(obj))
        for i, v in enumerate(obj):
            flatten(f"{prefix}.{i}", v, out)
    elif isinstance(obj, (list, tuple)) and (not obj or isinstance(obj[0], str)):
        out[prefix] = np.asarray(list(obj), dtype="U32")
        if not obj:
            out[f"{prefix}.count"] = np.int64(0)
    else:
        out[prefix] = np.asarray(obj)


def local_size(dom) -> int:
    return int(dom["ncomp"]) * int(dom["n_elements"]) * len(dom["l2g"]) // int(dom["n_elements"])


def solver_goldens(rd, solver, prob, out: dict, real) -> None:
    """Per-block forces, gather, assemble and internal forces on seeded inputs."""
    for di, dom in enumerate(prob["domains"]):
        nl = int(dom["ncomp"]) * len(dom["l2g"])
        ng = int(dom["ncomp"]) * int(dom["n_global"])
        u_local = np.random.default_rng(SEED_BLOCK + di).standard_normal(nl).astype(real)
        f_local = np.zeros(nl, real)
        for bi in range(len(dom["blocks"])):
            f = np.asarray(rd.block_forces(solver, di, bi, u_local))
            nz = f != 0
            f_local[nz] = f[nz]
            out[f"gold.d{di}.b{bi}.f_local"] = f
        out[f"gold.d{di}.f_local"] = f_local
        g = np.random.default_rng(SEED_GATHER + di).standard_normal(ng).astype(real)
        out[f"gold.d{di}.gather"] = np.asarray(rd.gather(solver, di, g))
        fl = np.random.default_rng(SEED_ASSEMBLE + di).standard_normal(nl).astype(real)
        out[f"gold.d{di}.assemble"] = np.asarray(rd.assemble(solver, di, fl))
        x = np.random.default_rng(SEED_FORCES + di).standard_normal(ng).astype(real)
        out[f"gold.d{di}.internal_forces"] = np.asarray(rd.internal_forces(solver, di, x))


def run_variant(variant: str, outdir: Path, only: list[str] | None) -> dict:
    sys.path.insert(0, str(REF_BUILD / variant))
    sys.path.insert(0, str(HERE))
    import insem  # noqa: F401  (the reference package, oracle build)
    import _refdump as rd
    import cases

    real = np.float64 if variant == "double" else np.float32
    summary = {}
    names = list(cases.RUN_CASES) + [f"blk{n}" for n in range(2, 10)]
    for name in names:
        if only and name not in only:
            continue
        out: dict = {}
        if name.startswith("blk"):
            sims = cases.blk(int(name[3:]))
            out["count"] = np.int64(len(sims))
            for si, sim in enumerate(sims):
                solver = sim.solver
                prob = rd.problem(solver)
                part: dict = {}
                flatten("problem", prob, part)
                solver_goldens(rd, solver, prob, part, real)
                for k, v in part.items():
                    out[f"m{si}.{k}"] = v
        else:
            sim, init = cases.RUN_CASES[name]()
            solver = sim.solver
            if init is not None:
                init(solver)
            prob = rd.problem(solver)
            flatten("problem", prob, out)
            for di in range(len(prob["domains"])):
                f = rd.fields(solver, di)
                out[f"init.d{di}.u"] = np.asarray(f["u"])
                out[f"init.d{di}.v"] = np.asarray(f["v"])
            solver_goldens(rd, solver, prob, out, real)
            # advance in two calls to pin the advance(n) semantics.
            first = solver.n_steps // 3
            solver.advance(first)
            solver.run()
            out["run.times"] = np.asarray(solver.times)
            for r in prob["receivers"]:
                for q in r["quantities"]:
                    out[f"run.trace.{r['name']}.{q}"] = np.asarray(solver.trace(r["name"], q))
            out["run.energy"] = np.asarray(solver.energy).reshape(-1, 3)
            for di in range(len(prob["domains"])):
                f = rd.fields(solver, di)
                for k in ("u", "v", "a"):
                    out[f"run.d{di}.{k}"] = np.asarray(f[k])
            out["run.advance_first"] = np.int64(first)
        if variant == "float":
            np.savez_compressed(outdir / f"{name}.npz", **out)
        elif variant == "double" and not name.startswith("blk"):
            keep = {k: v for k, v in out.items() if k.startswith("run.") or k in ("problem.dt", "problem.n_steps")}
            np.savez_compressed(outdir / f"{name}_f64.npz", **keep)
        elif variant == "strict":
            ref = np.load(outdir / f"{name}.npz")
            diffs = [k for k in out if (k.startswith("gold.") or k.startswith("run.") or ".gold." in k)
                     and not np.array_equal(np.asarray(ref[k]), np.asarray(out[k]))]
            summary[name] = {"strict_equals_float": not diffs, "differing": diffs[:5]}
        print(f"[{variant}] {name}: {len(out)} arrays", flush=True)
    return summary


def digest(a) -> str:
    a = np.ascontiguousarray(np.asarray(a))
    return hashlib.sha256(a.tobytes()).hexdigest()


TRACE_SAMPLES_KEPT = 600


def thin_traces(out: dict) -> dict:
    """Long runs: every trace keeps a SHA-256 digest of all its samples (the
    bitwise check) and every k-th sample row (the tolerance checks), k chosen
    so that about TRACE_SAMPLES_KEPT rows remain; the sample times likewise."""
    n = len(out["run.times"])
    stride = max(1, -(-n // TRACE_SAMPLES_KEPT))
    res = dict(out)
    res["meta.trace_stride"] = np.int64(stride)
    for k, v in out.items():
        if k.startswith("run.trace.") or k == "run.times":
            a = np.ascontiguousarray(np.asarray(v))
            res[f"hash.{k}"] = np.asarray(digest(a))
            res[f"shape.{k}"] = np.asarray(a.shape, np.int64)
            res[k] = a[::stride]
    return res


def run_timed_variant(variant: str, outdir: Path, only: list[str] | None) -> None:
    sys.path.insert(0, str(REF_BUILD / variant))
    sys.path.insert(0, str(HERE))
    sys.path.insert(0, str(REPO))
    import insem  # noqa: F401  (the reference package, oracle build)
    import _refdump as rd
    import timed_cases

    for name, make in timed_cases.TIMED_CASES.items():
        if only and name not in only:
            continue
        t_start = time.time()
        sim, n_run, model = make()
        if variant == "double":
            ref = np.load(outdir / f"timed_{name}.npz")
            sim.set_time(n_steps=model.n_steps, duration=model.duration, dt=float(ref["meta.dt"]),
                         safety=model.safety, record_every=model.record_every, energy_every=model.energy_every,
                         snapshot_every=model.snapshot_every, snapshot_quantities=list(model.snapshot_quantities))
        solver = sim.solver
        n_full = int(solver.n_steps)
        n_run = n_full if n_run <= 0 else min(n_run, n_full)
        out: dict = {"meta.n_steps_full": np.int64(n_full), "meta.n_steps_run": np.int64(n_run),
                     "meta.dt": np.float64(solver.dt), "meta.stable_dt": np.float64(solver.stable_dt)}
        if variant == "float":
            prob: dict = {}
            flatten("problem", rd.problem(solver), prob)
            for k, v in prob.items():
                a = np.asarray(v)
                if a.dtype.kind in "US":
                    out[f"text.{k}"] = a
                    continue
                out[f"hash.{k}"] = np.asarray(digest(a))
                out[f"dtype.{k}"] = np.asarray(a.dtype.str)
                out[f"size.{k}"] = np.int64(a.size)
        first = n_run // 3
        solver.advance(first)
        solver.advance(n_run - first)
        out["run.times"] = np.asarray(solver.times)
        for rec in model.receivers:
            for q in rec.quantities:
                out[f"run.trace.{rec.name}.{q}"] = np.asarray(solver.trace(rec.name, q))
        out["run.energy"] = np.asarray(solver.energy).reshape(-1, 3)
        if variant == "float" and model.snapshot_every > 0:
            out["snap.times"] = np.asarray(solver.snapshot_times)
            for medium in ("acoustic", "elastic"):
                for q in model.snapshot_quantities:
                    try:
                        a = np.ascontiguousarray(np.asarray(solver.snapshot(medium, q)))
                    except Exception:  # the medium does not have that quantity
                        continue
                    out[f"hash.snap.{medium}.{q}"] = np.asarray(digest(a))
                    out[f"shape.snap.{medium}.{q}"] = np.asarray(a.shape, np.int64)
                    out[f"norm.snap.{medium}.{q}"] = np.float64(np.linalg.norm(a.astype(np.float64)))
        if variant == "float":
            for di in range(len(rd.problem(solver)["domains"])):
                f = rd.fields(solver, di)
                for k in ("u", "v", "a"):
                    a = np.asarray(f[k])
                    out[f"hash.run.d{di}.{k}"] = np.asarray(digest(a))
                    out[f"norm.run.d{di}.{k}"] = np.float64(np.linalg.norm(a.astype(np.float64)))
        suffix = "" if variant == "float" else "_f64"
        np.savez_compressed(outdir / f"timed_{name}{suffix}.npz", **thin_traces(out))
        print(f"[{variant}] timed {name}: {n_run} of {n_full} steps, dt {solver.dt:.6e}, "
              f"{time.time() - t_start:.1f} s", flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--variant", choices=["float", "double", "strict"])
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--timed", action="store_true", help="fixtures of the benchmarked configurations")
    args = ap.parse_args()
    outdir = Path(args.out)
    if args.timed:
        if args.variant:
            run_timed_variant(args.variant, outdir, args.only)
            return
        env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1", OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
        for variant in ("float", "double"):
            cmd = [sys.executable, __file__, "--timed", "--variant", variant, "--out", str(outdir)]
            if args.only:
                cmd += ["--only", *args.only]
            subprocess.run(cmd, check=True, env=env)
        return
    if args.variant:
        summary = run_variant(args.variant, outdir, args.only)
        if summary:
            (outdir / "strict_check.json").write_text(json.dumps(summary, indent=1, sort_keys=True) + "\n")
        return
    env = dict(os.environ, PYTHONDONTWRITEBYTECODE="1", OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
    for variant in ("float", "double", "strict"):
        cmd = [sys.executable, __file__, "--variant", variant, "--out", str(outdir)]
        if args.only:
            cmd += ["--only", *args.only]
        subprocess.run(cmd, check=True, env=env)


if __name__ == "__main__":
    main()
