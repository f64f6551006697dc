"""Source-time functions of the reference, as FP32 tables for sfg_set_stf_table.

Ricker: factor * (1 - 2 a t^2) exp(-a t^2) (core/specfem/source_time_functions/ricker.cpp,
impl/time_functions.hpp:78); Dirac: factor * (-exp(-a t^2) / (2 a)) with
f0 = 1/(10 dt) (dirac.cpp:25, time_functions.hpp gaussian); a = pi^2 f0^2 and
t = t0 + i dt - tshift, where t0 is the earliest source start -1.2/f0 + tshift
and each source's shift becomes its own start minus t0
(src/io/sources/dim2/read_sources.cpp:142-172).
"""
from __future__ import annotations

import numpy as np


def table(sources, dt: float, nstep: int) -> np.ndarray:
    """[nstep, nsrc] float32 table of the sources' time functions (one shot)."""
    f32 = np.float32
    f0 = [f32(1.0) / (f32(10.0) * f32(dt)) if getattr(s, "stf", "ricker") == "dirac" else f32(s.f0)
          for s in sources]
    starts = [f32(-1.2) * (f32(1.0) / f) + f32(getattr(s, "tshift", 0.0)) for s, f in zip(sources, f0)]
    t0 = min(starts)
    i = np.arange(nstep, dtype=f32)
    out = np.zeros((nstep, len(sources)), np.float32)
    pi = f32(np.pi)
    for k, s in enumerate(sources):
        t = f32(t0) + i * f32(dt) - f32(starts[k] - t0)
        a = pi * pi * f0[k] * f0[k]
        if getattr(s, "stf", "ricker") == "dirac":
            out[:, k] = f32(s.factor) * (f32(-1.0) * np.exp(-a * t * t) / (f32(2.0) * a))
        else:
            out[:, k] = f32(s.factor) * ((f32(1.0) - f32(2.0) * a * t * t) * np.exp(-a * t * t))
    return out
