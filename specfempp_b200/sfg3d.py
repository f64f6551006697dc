"""ctypes binding of the 3D interface of libsfg (``include/sfg3d.h``).

Structured hexahedral meshes (``meshgen.Mesh3D``), isotropic elastic media
per GLL point, force and moment-tensor sources, receivers; the CUDA library
must be built, there is no fallback path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .sfg import ERRORS, SEIS, SfgError, Options, load_library

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class MeshDesc3D(C.Structure):
    _fields_ = [("nex", C.c_int), ("ney", C.c_int), ("nez", C.c_int), ("nodes", _dp),
                ("rho", _fp), ("vp", _fp), ("vs", _fp), ("absorbing", C.c_int * 6)]


class SourceDesc3D(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double), ("kind", C.c_int), ("stf", C.c_int),
                ("f0", C.c_double), ("factor", C.c_double), ("tshift", C.c_double), ("comp", C.c_double * 6)]


class Info3D(C.Structure):
    _fields_ = [("nspec", C.c_int), ("nglob", C.c_int), ("nstep", C.c_int), ("istep", C.c_int),
                ("nrec", C.c_int), ("ntypes", C.c_int), ("nsig", C.c_int), ("nsrc", C.c_int),
                ("t0", C.c_double), ("device_bytes", C.c_size_t), ("elements_per_block", C.c_int),
                ("kernels_per_step", C.c_int), ("kernel_variant", C.c_int)]


_vp = C.c_void_p
EXPORTS3D = {
    "sfg3d_create": ([C.POINTER(MeshDesc3D), C.POINTER(Options), C.POINTER(_vp)], C.c_int),
    "sfg3d_destroy": ([_vp], None),
    "sfg3d_last_error": ([_vp], C.c_char_p),
    "sfg3d_set_sources": ([_vp, C.c_int, C.POINTER(SourceDesc3D)], C.c_int),
    "sfg3d_set_receivers": ([_vp, C.c_int, _dp, C.c_int, _ip], C.c_int),
    "sfg3d_initialize": ([_vp], C.c_int),
    "sfg3d_run": ([_vp, C.c_int], C.c_int),
    "sfg3d_run_timed": ([_vp, C.c_int, _fp], C.c_int),
    "sfg3d_run_timed_flushed": ([_vp, C.c_int, C.c_size_t, _fp], C.c_int),
    "sfg3d_step_io": ([_vp, _fp, _fp], C.c_int),
    "sfg3d_time_kernel": ([_vp, C.c_int, C.c_int, _fp], C.c_int),
    "sfg3d_reset_fields": ([_vp], C.c_int),
    "sfg3d_get_info": ([_vp, C.POINTER(Info3D)], C.c_int),
    "sfg3d_get_seismograms": ([_vp, _fp, C.c_size_t], C.c_int),
    "sfg3d_get_field": ([_vp, C.c_int, _fp, C.c_size_t], C.c_int),
    "sfg3d_check_finite": ([_vp], C.c_int),
}


def load_library3d():
    lib = load_library()
    if not getattr(lib, "_sfg3d_declared", False):
        for name, (args, res) in EXPORTS3D.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        lib._sfg3d_declared = True
    return lib


def _arr(x, dtype):
    return np.ascontiguousarray(x, dtype=dtype)


class Simulation3D:
    """One 3D elastic forward simulation on the GPU (a libsfg 3D handle)."""

    def __init__(self, mesh, *, dt: float, nstep: int, elements_per_block: int = 0, steps_per_graph: int = 0,
                 kernel_variant: int = 0):
        self.lib = load_library3d()
        self._keep = []
        d = MeshDesc3D()
        d.nex, d.ney, d.nez = mesh.nex, mesh.ney, mesh.nez
        nodes = _arr(mesh.nodes, np.float64)
        rho, vp, vs = (_arr(a, np.float32) for a in (mesh.rho, mesh.vp, mesh.vs))
        self._keep += [nodes, rho, vp, vs]
        d.nodes = nodes.ctypes.data_as(_dp)
        d.rho, d.vp, d.vs = (a.ctypes.data_as(_fp) for a in (rho, vp, vs))
        for i in range(6):
            d.absorbing[i] = int(mesh.absorbing[i])
        o = Options(dt=dt, nstep=nstep, nshots=1, nstep_between_samples=1, steps_per_graph=steps_per_graph,
                    elements_per_block=elements_per_block, kernel_variant=kernel_variant, store_acceleration=0)
        h = _vp()
        rc = self.lib.sfg3d_create(C.byref(d), C.byref(o), C.byref(h))
        if rc != 0:
            raise SfgError(rc, self.lib.sfg3d_last_error(None).decode())
        self.h = h
        self.nstep = nstep

    def _check(self, rc):
        if rc != 0:
            raise SfgError(rc, self.lib.sfg3d_last_error(self.h).decode())

    def set_sources(self, sources):
        arr = (SourceDesc3D * len(sources))()
        for i, s in enumerate(sources):
            comp = (C.c_double * 6)(*[float(c) for c in s.comp])
            arr[i] = SourceDesc3D(x=s.x, y=s.y, z=s.z, kind=1 if s.kind == "moment_tensor" else 0, stf=0,
                                  f0=s.f0, factor=s.factor, tshift=getattr(s, "tshift", 0.0), comp=comp)
        self._check(self.lib.sfg3d_set_sources(self.h, len(sources), arr))

    def set_receivers(self, xyz, types=("displacement",)):
        xyz = _arr(xyz, np.float64)
        ty = _arr([SEIS[t] for t in types], np.int32)
        self._check(self.lib.sfg3d_set_receivers(self.h, len(xyz), xyz.ctypes.data_as(_dp), len(ty),
                                                 ty.ctypes.data_as(_ip)))

    def initialize(self):
        self._check(self.lib.sfg3d_initialize(self.h))

    def run(self, nsteps):
        self._check(self.lib.sfg3d_run(self.h, int(nsteps)))

    def run_timed(self, nsteps) -> float:
        ms = C.c_float()
        self._check(self.lib.sfg3d_run_timed(self.h, int(nsteps), C.byref(ms)))
        return ms.value

    def run_timed_flushed(self, nsteps, flush_bytes=256 << 20) -> float:
        ms = C.c_float()
        self._check(self.lib.sfg3d_run_timed_flushed(self.h, int(nsteps), flush_bytes, C.byref(ms)))
        return ms.value

    def step_io(self, stf_row, seis_row):
        self._check(self.lib.sfg3d_step_io(self.h, stf_row.ctypes.data_as(_fp) if stf_row is not None else None,
                                           seis_row.ctypes.data_as(_fp) if seis_row is not None else None))

    def time_kernel(self, which, reps=20) -> float:
        ms = C.c_float()
        self._check(self.lib.sfg3d_time_kernel(self.h, int(which), int(reps), C.byref(ms)))
        return ms.value

    def reset(self):
        self._check(self.lib.sfg3d_reset_fields(self.h))

    def info(self) -> Info3D:
        inf = Info3D()
        self._check(self.lib.sfg3d_get_info(self.h, C.byref(inf)))
        return inf

    def seismograms(self) -> np.ndarray:
        """[nstep, ntypes, nrec, 3] float32."""
        i = self.info()
        out = np.zeros((i.nsig, i.ntypes, i.nrec, 3), np.float32)
        self._check(self.lib.sfg3d_get_seismograms(self.h, out.ctypes.data_as(_fp), out.size))
        return out

    def field(self, which="displacement") -> np.ndarray:
        i = self.info()
        out = np.zeros((i.nglob, 3), np.float32)
        self._check(self.lib.sfg3d_get_field(self.h, {"displacement": 0, "velocity": 1, "acceleration": 2}[which],
                                             out.ctypes.data_as(_fp), out.size))
        return out

    def check_finite(self) -> bool:
        return self.lib.sfg3d_check_finite(self.h) == 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfg3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
