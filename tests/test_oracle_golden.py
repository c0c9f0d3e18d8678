"""The oracle against the reference's own outputs (CPU only).

Pins the C restatement (oracle/insem_oracle.c) before it is trusted as the
checker: every per-block force vector, gather, assemble and internal-force
golden, and full runs (traces, sample times, final fields, energy), must match
the reference float build bit for bit.  The reference double build (FP64
oracle) is compared with tolerances to state the float path's error.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import BLK_CASES, RUN_CASES, golden
import golden_io as G


def bits(a):
    return np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32)


@pytest.mark.parametrize("case", RUN_CASES + BLK_CASES)
def test_oracle_kernels_bitwise(pkg, oracle, case):
    z = golden(case)
    for prefix, prob in G.sub_problems(pkg, z):
        for di, d in enumerate(prob.domains):
            u = G.block_input(d, di)
            for bi in range(len(d.blocks)):
                f = oracle.block_forces(prob, di, bi, u)
                assert np.array_equal(bits(f), bits(z[f"{prefix}gold.d{di}.b{bi}.f_local"])), (case, prefix, di, bi)
            assert np.array_equal(bits(oracle.gather(prob, di, G.gather_input(d, di))),
                                  bits(z[f"{prefix}gold.d{di}.gather"]))
            assert np.array_equal(bits(oracle.assemble(prob, di, G.assemble_input(d, di))),
                                  bits(z[f"{prefix}gold.d{di}.assemble"]))
        s = oracle.OracleSolver(prob)
        for di, d in enumerate(prob.domains):
            f = s.internal_forces(di, G.forces_input(d, di))
            assert np.array_equal(bits(f), bits(z[f"{prefix}gold.d{di}.internal_forces"]))


def oracle_run(pkg, oracle, z):
    prob = pkg.ProblemData.from_npz(z)
    s = oracle.OracleSolver(prob)
    for di in range(len(prob.domains)):
        u0, v0 = z[f"init.d{di}.u"], z[f"init.d{di}.v"]
        if np.any(u0) or np.any(v0):
            s.set_state(prob.media[di], u0.astype(np.float64), v0.astype(np.float64))
    s.advance(int(z["run.advance_first"]))
    s.run()
    return prob, s


@pytest.mark.parametrize("case", RUN_CASES)
def test_oracle_run_bitwise(pkg, oracle, case):
    z = golden(case)
    prob, s = oracle_run(pkg, oracle, z)
    assert s.step == prob.n_steps
    for name, q in prob.trace_list():
        assert np.array_equal(s.trace(name, q), z[f"run.trace.{name}.{q}"]), (case, name, q)
    for di in range(len(prob.domains)):
        for k, arr in zip("uva", s.state(di)):
            assert np.array_equal(arr.ravel(), z[f"run.d{di}.{k}"].astype(np.float64)), (case, di, k)
    assert np.array_equal(s.energy, z["run.energy"])


@pytest.mark.parametrize("case", RUN_CASES)
def test_float_vs_double_reference(pkg, case):
    """States the float path's error against the FP64 reference build (not a pass/fail of parity:
    the bound only guards against a broken fixture)."""
    z, z64 = golden(case), golden(f"{case}_f64")
    prob = pkg.ProblemData.from_npz(z)
    for name, q in prob.trace_list():
        a, b = z[f"run.trace.{name}.{q}"], z64[f"run.trace.{name}.{q}"]
        assert a.shape == b.shape
        assert G.rel_l2(a, b) < 5e-2, (case, name, q, G.rel_l2(a, b))
