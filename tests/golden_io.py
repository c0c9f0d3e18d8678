"""Readers for the golden fixtures (tests/golden/*.npz, made by make_golden.py).

Random inputs of the per-block, gather, assemble and internal-force goldens
are regenerated here from the generator's seeds; outputs come from the files.
"""

from __future__ import annotations

from typing import Iterator, Tuple

import numpy as np

SEED_BLOCK = 101
SEED_GATHER = 202
SEED_ASSEMBLE = 303
SEED_FORCES = 404


def sub_problems(pkg, z) -> Iterator[Tuple[str, object]]:
    """(prefix, ProblemData) of every model in a fixture (blk files hold several)."""
    if "count" in z.files:
        for m in range(int(z["count"])):
            yield f"m{m}.", pkg.ProblemData.from_npz(z, prefix=f"m{m}.problem.")
    else:
        yield "", pkg.ProblemData.from_npz(z)


def block_input(d, di: int) -> np.ndarray:
    nl = d.ncomp * d.l2g.size
    return np.random.default_rng(SEED_BLOCK + di).standard_normal(nl).astype(np.float32)


def gather_input(d, di: int) -> np.ndarray:
    return np.random.default_rng(SEED_GATHER + di).standard_normal(d.ncomp * d.n_global).astype(np.float32)


def assemble_input(d, di: int) -> np.ndarray:
    return np.random.default_rng(SEED_ASSEMBLE + di).standard_normal(d.ncomp * d.l2g.size).astype(np.float32)


def forces_input(d, di: int) -> np.ndarray:
    return np.random.default_rng(SEED_FORCES + di).standard_normal(d.ncomp * d.n_global).astype(np.float32)


def rel_l2(a, b) -> float:
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))
