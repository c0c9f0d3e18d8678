"""Tile-size autotuner of the tiled step.

A tile is one CTA of ``te`` elements, with one thread per element column.
Its best size depends on the class:
- ngll, geometry kind, medium and azimuthal order set the shared memory per
  element and the registers per thread;
- the element count per tile sets how many CTAs stay resident per SM, and
  how many points each tile shares with its neighbours (halo work).

The library starts from an occupancy-based choice. This module times
candidate sizes around that choice on real problems, one class at a time,
with the other classes held: ``tune`` on solo solves, ``tune_batched`` on the
tile launches of a batch of the class's largest problems (the setting of the
batched workload). It keeps the fastest and registers it
process-wide (``insem_cuda_set_tile_elements``), so solvers built afterwards
use it. Tables can be saved as JSON and loaded again.
"""

from __future__ import annotations

import json
from typing import Dict, Iterable, List, Optional, Tuple

from . import native as N
from .problem import ProblemData
from .solver import Solver

ClassKey = Tuple[int, int, int, int, int]  # ngll, kind, medium, azimuthal order, ncomp


def te_max(ngll: int) -> int:
    return min(64, 256 // ngll)


def current(key: ClassKey) -> int:
    ngll, kind, medium, m, ncomp = key
    return int(N.lib().insem_cuda_tile_elements(ngll, kind, medium, m, ncomp))


def register(key: ClassKey, te: int) -> None:
    ngll, kind, medium, m, _ = key
    N.check(N.lib().insem_cuda_set_tile_elements(ngll, kind, medium, m if kind == N.AXISYM else 0, int(te)))


def classes_of(problem: ProblemData) -> List[ClassKey]:
    """The tile class of every domain: its dominant element kind decides."""
    out = []
    for d in problem.domains:
        count: Dict[int, int] = {}
        for b in d.blocks:
            count[b.kind] = count.get(b.kind, 0) + b.n_elements
        kind = max(count.items(), key=lambda kv: kv[1])[0]
        out.append((problem.ngll, kind, d.medium, d.azimuthal_order if kind == N.AXISYM else 0, d.ncomp))
    return out


def candidates(key: ClassKey) -> List[int]:
    base = current(key)
    hi = te_max(key[0])
    vals = {base, hi, max(1, round(base * 1.5)), max(1, round(base / 1.5)), max(1, base // 2)}
    return sorted(v for v in vals if 1 <= v <= hi)


def time_problem(problem: ProblemData, device: int, warmup: int, steps: int) -> float:
    """Device ms per step of a fresh solver (graphs), after warm-up."""
    with Solver(problem, device=device) as s:
        s.advance(warmup)
        s.advance(steps)
        return s.last_advance_ms / steps


def tune(problems: Iterable[ProblemData], device: int = 0, warmup: int = 3, steps: int = 20,
         verbose: bool = False) -> Dict[ClassKey, dict]:
    """Tunes every class of the given problems on the first (largest) problem
    of each class; registers and returns {class: {te, ms, timings}}."""
    reps: Dict[ClassKey, ProblemData] = {}
    for p in problems:
        for key in classes_of(p):
            if key not in reps or p.n_elements_total() > reps[key].n_elements_total():
                reps[key] = p
    out: Dict[ClassKey, dict] = {}
    for key, prob in sorted(reps.items()):
        timings = {}
        for te in candidates(key):
            register(key, te)
            timings[te] = time_problem(prob, device, warmup, steps)
            if verbose:
                print(f"  class {key} te={te}: {timings[te]:.4f} ms/step", flush=True)
        best = min(timings, key=timings.get)
        register(key, best)
        out[key] = {"te": best, "ms": timings[best], "timings": timings}
    return out


def tune_batched(problems: Iterable[ProblemData], device: int = 0, reps: int = 2, warmup: int = 3, steps: int = 6,
                 min_share: float = 0.05, verbose: bool = False) -> Dict[ClassKey, dict]:
    """Tunes the classes that hold at least `min_share` of the problems'
    elements, in the setting they run in: the `reps` largest problems of the
    class are built into a batch at every candidate size, and the batch's
    tile launches are timed with CUDA events (Batch.profile).  The other
    classes keep their current choice.  Registers and returns the choices."""
    from .batch import Batch

    problems = list(problems)
    weight: Dict[ClassKey, int] = {}
    members: Dict[ClassKey, List[ProblemData]] = {}
    for p in problems:
        for key, d in zip(classes_of(p), p.domains):
            weight[key] = weight.get(key, 0) + d.n_elements
            members.setdefault(key, []).append(p)
    total = sum(weight.values()) or 1
    out: Dict[ClassKey, dict] = {}
    for key in sorted(weight, key=lambda k: -weight[k]):
        if weight[key] < min_share * total:
            continue
        group = sorted(members[key], key=lambda p: -p.n_elements_total())[:reps]
        timings = {}
        for te in candidates(key):
            register(key, te)
            with Batch(device=device) as b:
                for prob in group:
                    b.adopt(Solver(prob, device=device))
                b.advance(warmup)
                tile_ms, _ = b.profile(steps)
            timings[te] = tile_ms / steps
            if verbose:
                print(f"  class {key} te={te}: {timings[te]:.4f} ms of tile launches per step", flush=True)
        best = min(timings, key=timings.get)
        register(key, best)
        out[key] = {"te": best, "ms": timings[best], "timings": timings, "share": weight[key] / total}
    return out


def save(table: Dict[ClassKey, dict], path: str) -> None:
    rows = [{"class": list(k), "te": v["te"], "ms": v.get("ms"), "timings": v.get("timings")} for k, v in table.items()]
    with open(path, "w") as f:
        json.dump({"tiles": rows}, f, indent=1)


def load(path: str) -> Dict[ClassKey, dict]:
    """Reads a saved table and registers every entry."""
    with open(path) as f:
        rows = json.load(f)["tiles"]
    out = {}
    for r in rows:
        key = tuple(r["class"])
        register(key, r["te"])
        out[key] = {"te": r["te"], "ms": r.get("ms")}
    return out


def summary(table: Optional[Dict[ClassKey, dict]]) -> list:
    if not table:
        return []
    names = {N.RECT: "rect", N.AFFINE: "affine", N.CURVED: "curved", N.AXISYM: "axisym"}
    return [{"ngll": k[0], "kind": names.get(k[1], k[1]), "medium": "elastic" if k[2] == N.ELASTIC else "acoustic",
             "m": k[3], "te": v["te"], "ms_per_step": round(v["ms"], 5),
             **({"share": round(v["share"], 3)} if "share" in v else {})} for k, v in sorted(table.items())]
