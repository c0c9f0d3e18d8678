"""Source time functions on the host (SourceTimeFunction::operator(),
cpp/src/sim/description.cpp:88-113), evaluated with the C library's exp so the
per-step amplitudes (real_t)stf(step * dt) equal the reference's."""

from __future__ import annotations

import math

import numpy as np


def value(kind: int, f0: float, t0: float, amplitude: float, t: float, samples=None, sample_dt: float = 0.0) -> float:
    if kind == 0:
        x = math.pi * f0 * (t - t0)
        a = x * x
        return amplitude * (1.0 - 2.0 * a) * math.exp(-a)
    if kind == 1:
        x = math.pi * f0 * (t - t0)
        return amplitude * math.exp(-(x * x))
    if kind == 2:
        tau = t - t0
        y = math.pi * f0
        c = y * y
        return amplitude * (-2.0 * c * tau) * math.exp(-c * tau * tau)
    if samples is None or len(samples) == 0:
        return 0.0
    x = t / sample_dt
    if x < 0.0 or x > len(samples) - 1:
        return 0.0
    i = int(x)
    if i + 1 >= len(samples):
        return amplitude * samples[-1]
    w = x - i
    return amplitude * ((1.0 - w) * samples[i] + w * samples[i + 1])


def amplitudes(problem, first_step: int, n: int) -> np.ndarray:
    """[n][n_sources] float32 amplitudes of steps first_step .. first_step + n - 1."""
    out = np.zeros((n, len(problem.sources)), np.float32)
    for q, s in enumerate(problem.sources):
        for k in range(n):
            t = (first_step + k) * problem.dt
            out[k, q] = value(s.stf_kind, s.f0, s.t0, s.amplitude, t, s.samples, s.sample_dt)
    return out
