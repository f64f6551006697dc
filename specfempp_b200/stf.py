"""Source-time functions of the reference, as FP32 tables for sfg_set_stf_table.

The same tables the library builds in sfg_set_sources (FP32 like the
reference's; core/specfem/source_time_functions/impl/time_functions.hpp):
  ricker         factor (1 - 2 a t^2) exp(-a t^2)              (ricker.cpp)
  dirac          factor (-exp(-a t^2) / (2 a)), f0 = 1/(10 dt)  (dirac.cpp:25)
  gaussian       factor (-exp(-a t^2) / (2 a))                  (gaussian.cpp)
  dgaussian      factor t exp(-a t^2)                           (dgaussian.cpp)
  gaussian_hdur  factor exp(-t^2 / h^2) / (sqrt(pi) h)          (gaussianhdur.cpp)
  heaviside      factor (1 + erf(t / h)) / 2                    (heaviside.cpp)
with a = pi^2 f0^2.  Start times: -1.2/f0 + tshift (ricker, dirac, dgaussian),
-2/f0 + tshift (gaussian), -2 hdur + tshift with hdur raised to 5 dt and
h = hdur / 1.628 (gaussian_hdur, heaviside).  t = t0 + i dt - shift, where t0
is the earliest start and each source's shift is its start minus t0
(src/io/sources/dim2/read_sources.cpp:142-172).
"""
from __future__ import annotations

import math

import numpy as np

_f32 = np.float32


def start(s, dt: float):
    """(start time, evaluation parameter f0 or h) of one source, FP32."""
    kind = getattr(s, "stf", "ricker")
    tshift = _f32(getattr(s, "tshift", 0.0))
    if kind in ("gaussian_hdur", "heaviside"):
        hd = max(_f32(s.hdur), _f32(5.0) * _f32(dt))
        return _f32(_f32(-2.0) * hd + tshift), _f32(hd / _f32(1.628))
    f0 = _f32(1.0) / (_f32(10.0) * _f32(dt)) if kind == "dirac" else _f32(s.f0)
    fac = _f32(2.0) if kind == "gaussian" else _f32(1.2)
    return _f32(-fac * (_f32(1.0) / f0) + tshift), f0


def values(kind: str, t: np.ndarray, p, factor) -> np.ndarray:
    """FP32 values of one time function at times t (p: f0 or h)."""
    t = t.astype(_f32)
    fac = _f32(factor)
    if kind in ("gaussian_hdur", "heaviside"):
        h = _f32(p)
        if kind == "heaviside":
            erf = np.array([math.erf(float(x)) for x in (t / h)], dtype=_f32)
            return fac * (_f32(0.5) * (_f32(1.0) + erf))
        ah = _f32(1.0) / (h * h)
        return fac * (np.exp(-ah * t * t) / (_f32(math.sqrt(math.pi)) * h))
    a = _f32(np.pi) * _f32(np.pi) * _f32(p) * _f32(p)
    if kind in ("dirac", "gaussian"):
        return fac * (_f32(-1.0) * np.exp(-a * t * t) / (_f32(2.0) * a))
    if kind == "dgaussian":
        return fac * (t * np.exp(-a * t * t))
    return fac * ((_f32(1.0) - _f32(2.0) * a * t * t) * np.exp(-a * t * t))


def table(sources, dt: float, nstep: int, start_time: float | None = None) -> np.ndarray:
    """[nstep, nsrc] float32 table of the sources' time functions (one shot);
    with ``start_time`` the run starts there and each source keeps its own
    tshift (read_sources.cpp:155-161)."""
    st = [start(s, dt) for s in sources]
    t0 = min(t for t, _ in st)
    shifts = [_f32(a - t0) for a, _ in st]
    if start_time is not None:
        t0 = _f32(start_time)
        shifts = [_f32(getattr(s, "tshift", 0.0)) for s in sources]
    i = np.arange(nstep, dtype=_f32)
    out = np.zeros((nstep, len(sources)), np.float32)
    for k, s in enumerate(sources):
        t = _f32(t0) + i * _f32(dt) - shifts[k]
        out[:, k] = values(getattr(s, "stf", "ricker"), t, st[k][1], s.factor)
    return out
