"""specfempp_b200 — B200-native (sm_100a) spectral-element time stepping.

The hot path of SPECFEM++ (per-step stiffness, Newmark, Stacey, coupling,
sources, seismograms) runs in hand-written CUDA behind the C ABI declared in
``include/sfg.h``; this package holds the C++/CUDA sources (``csrc/``), the
ctypes binding (``sfg.py``) and the structured-mesh generator (``meshgen.py``).
"""
from .sfg import Simulation2D, Source, SfgError, load_library  # noqa: F401

__all__ = ["Simulation2D", "Source", "SfgError", "load_library"]
