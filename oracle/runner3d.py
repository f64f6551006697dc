"""ctypes driver of the 3D CPU oracle (oracle3d.cpp) — test infrastructure.

Only tests/, the smoke check and bench.py's CPU-baseline leg use it, as the
checker of the CUDA path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from .runner import lib

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
SEIS_TYPES = {"displacement": 0, "velocity": 1, "acceleration": 2}


class OracleInput3D(C.Structure):
    _fields_ = [
        ("nex", C.c_int), ("ney", C.c_int), ("nez", C.c_int),
        ("nodes", _dp), ("rho", _dp), ("vp", _dp), ("vs", _dp),
        ("absorbing", C.c_int * 6),
        ("nsrc", C.c_int), ("src_kind", _ip), ("src_xyz", _dp), ("src_comp", _dp),
        ("src_f0", _dp), ("src_factor", _dp), ("src_tshift", _dp), ("t0", C.c_double),
        ("nrec", C.c_int), ("rec_xyz", _dp),
        ("ntypes", C.c_int), ("seis_types", _ip),
        ("dt", C.c_double), ("nstep", C.c_int), ("device_order", C.c_int),
    ]


class OracleOutput3D(C.Structure):
    _fields_ = [("seismograms", _dp), ("final_u", _dp), ("nglob", C.c_int), ("seconds", C.c_double),
                ("error", C.c_char * 256)]


@dataclass
class Source3D:
    x: float
    y: float
    z: float
    f0: float
    factor: float
    kind: str = "force"                 # "force" or "moment_tensor"
    comp: tuple = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0)  # (fx, fy, fz, ...) or (Mxx, Myy, Mzz, Mxy, Mxz, Myz)
    tshift: float = 0.0


@dataclass
class Case3D:
    mesh: object                        # nex, ney, nez, nodes, rho, vp, vs, absorbing
    sources: list
    rec_xyz: np.ndarray
    dt: float
    nstep: int
    seis_types: list = field(default_factory=lambda: ["displacement"])
    device_order: bool = False          # True: FMA contractions as the CUDA kernels evaluate them


def start_time(sources):
    """t0 = min over sources of -1.2/f0 + tshift (read_sources.cpp:142-172);
    each source's shift becomes its own start minus t0."""
    t = [np.float32(-1.2) * (np.float32(1.0) / np.float32(s.f0)) + np.float32(s.tshift) for s in sources]
    t0 = float(min(t))
    return t0, [float(ti) - t0 for ti in t]


def run(case: Case3D, precision: str = "f32", nthreads: int = 8, want_final: bool = False):
    m = case.mesh
    L = lib()
    keep = []

    def arr(x, dt):
        a = np.ascontiguousarray(x, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(_dp if dt == np.float64 else _ip)

    inp = OracleInput3D()
    inp.nex, inp.ney, inp.nez = m.nex, m.ney, m.nez
    inp.nodes = arr(m.nodes, np.float64)
    inp.rho, inp.vp, inp.vs = arr(m.rho, np.float64), arr(m.vp, np.float64), arr(m.vs, np.float64)
    for i in range(6):
        inp.absorbing[i] = int(m.absorbing[i])
    t0, tsh = start_time(case.sources)
    inp.nsrc = len(case.sources)
    inp.src_kind = arr([1 if s.kind == "moment_tensor" else 0 for s in case.sources], np.int32)
    inp.src_xyz = arr([[s.x, s.y, s.z] for s in case.sources], np.float64)
    inp.src_comp = arr([list(s.comp) for s in case.sources], np.float64)
    inp.src_f0 = arr([s.f0 for s in case.sources], np.float64)
    inp.src_factor = arr([s.factor for s in case.sources], np.float64)
    inp.src_tshift = arr(tsh, np.float64)
    inp.t0 = t0
    inp.nrec = len(case.rec_xyz)
    inp.rec_xyz = arr(case.rec_xyz, np.float64)
    types = [SEIS_TYPES[t] for t in case.seis_types]
    inp.ntypes = len(types)
    inp.seis_types = arr(types, np.int32)
    inp.dt, inp.nstep = case.dt, case.nstep
    inp.device_order = int(case.device_order)
    seis = np.zeros((case.nstep, len(types), len(case.rec_xyz), 3))
    out = OracleOutput3D()
    out.seismograms = seis.ctypes.data_as(_dp)
    final = None
    if want_final:
        n = (4 * m.nex + 1) * (4 * m.ney + 1) * (4 * m.nez + 1)
        final = np.zeros((n, 3))
        out.final_u = final.ctypes.data_as(_dp)
    fn = L.oracle3d_run_f32 if precision == "f32" else L.oracle3d_run_f64
    fn.argtypes = [C.POINTER(OracleInput3D), C.POINTER(OracleOutput3D), C.c_int]
    fn.restype = C.c_int
    rc = fn(C.byref(inp), C.byref(out), nthreads)
    if rc != 0:
        raise RuntimeError(out.error.decode())
    return {"seis": seis, "t0": t0, "final": final, "nglob": out.nglob, "loop_seconds": out.seconds}
