"""ctypes binding of libsfg (``include/sfg.h``).

This is the Python face of the drop-in boundary: it passes plain host arrays
through the C ABI and gets seismograms and wavefields back as numpy arrays.
The CUDA library must be built (``__graft_entry__.build()`` or
``python -m specfempp_b200.build``); there is no fallback path — a missing
library raises ``ImportError`` when a simulation is created.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsfg.so")

SFG_MEDIUM_ACOUSTIC, SFG_MEDIUM_ELASTIC = 0, 1
SEIS = {"displacement": 0, "velocity": 1, "acceleration": 2, "pressure": 3, "rotation": 4,
        "intrinsic_rotation": 5, "curl": 6}
STF = {"ricker": 0, "dirac": 1, "gaussian": 2, "gaussian_hdur": 3, "dgaussian": 4, "heaviside": 5}
FIELD = {"displacement": 0, "velocity": 1, "acceleration": 2}
ERRORS = {0: "OK", -1: "SFG_ERR_ARG", -2: "SFG_ERR_IO", -3: "SFG_ERR_CUDA", -4: "SFG_ERR_LOCATE",
          -5: "SFG_ERR_STATE", -6: "SFG_ERR_NONFINITE", -7: "SFG_ERR_UNSUPPORTED"}

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class MeshDesc(C.Structure):
    _fields_ = [
        ("nspec", C.c_int), ("npgeo", C.c_int), ("ngnod", C.c_int),
        ("coorg", _dp), ("knods", _ip), ("kmato", _ip), ("numat", C.c_int),
        ("mat_medium", _ip), ("mat_rho", _dp), ("mat_vp", _dp), ("mat_vs", _dp),
        ("point_rho", _fp), ("point_vp", _fp), ("point_vs", _fp),
        ("nabs", C.c_int), ("abs_ispec", _ip), ("abs_type", _ip),
        ("nfree", C.c_int), ("free_ispec", _ip), ("free_type", _ip),
        ("elastic_wave", C.c_int),
        ("mat_aniso", _dp), ("mat_cosserat", _dp),
        ("nadj", C.c_int), ("adjacency", _ip), ("mat_poro", _dp),
    ]


class Options(C.Structure):
    _fields_ = [("dt", C.c_double), ("nstep", C.c_int), ("nshots", C.c_int),
                ("nstep_between_samples", C.c_int), ("steps_per_graph", C.c_int),
                ("elements_per_block", C.c_int), ("kernel_variant", C.c_int),
                ("store_acceleration", C.c_int), ("has_start_time", C.c_int), ("start_time", C.c_double)]


class Source2D(C.Structure):
    _fields_ = [("x", C.c_double), ("z", C.c_double), ("shot", C.c_int), ("stf", C.c_int),
                ("f0", C.c_double), ("factor", C.c_double), ("tshift", C.c_double),
                ("angle", C.c_double), ("kind", C.c_int), ("mxx", C.c_double), ("mzz", C.c_double),
                ("mxz", C.c_double), ("hdur", C.c_double)]


class Info(C.Structure):
    _fields_ = [("nspec", C.c_int), ("nspec_elastic", C.c_int), ("nspec_acoustic", C.c_int),
                ("nglob", C.c_int), ("nglob_elastic", C.c_int), ("nglob_acoustic", C.c_int),
                ("ncolors_elastic", C.c_int), ("ncolors_acoustic", C.c_int),
                ("nshots", C.c_int), ("nsig", C.c_int), ("nrec", C.c_int), ("ntypes", C.c_int),
                ("nstep", C.c_int), ("istep", C.c_int), ("t0", C.c_double),
                ("device_bytes", C.c_size_t), ("kernels_per_step", C.c_int),
                ("elements_per_block", C.c_int), ("kernel_variant", C.c_int), ("ncomp_elastic", C.c_int)]


EXPORTS = {
    "sfg_create2d": ([C.POINTER(MeshDesc), C.POINTER(Options), C.POINTER(C.c_void_p)], C.c_int),
    "sfg_create2d_from_database": ([C.c_char_p, C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)], C.c_int),
    "sfg_destroy": ([C.c_void_p], None),
    "sfg_last_error": ([C.c_void_p], C.c_char_p),
    "sfg_set_sources": ([C.c_void_p, C.c_int, C.POINTER(Source2D)], C.c_int),
    "sfg_set_stf_table": ([C.c_void_p, _fp, C.c_int, C.c_int], C.c_int),
    "sfg_set_receivers": ([C.c_void_p, C.c_int, _dp, _dp, C.c_double, C.c_int, _ip], C.c_int),
    "sfg_initialize": ([C.c_void_p], C.c_int),
    "sfg_step": ([C.c_void_p], C.c_int),
    "sfg_run": ([C.c_void_p, C.c_int], C.c_int),
    "sfg_synchronize": ([C.c_void_p], C.c_int),
    "sfg_reset_fields": ([C.c_void_p], C.c_int),
    "sfg_run_timed": ([C.c_void_p, C.c_int, _fp], C.c_int),
    "sfg_run_timed_flushed": ([C.c_void_p, C.c_int, C.c_size_t, _fp], C.c_int),
    "sfg_step_io": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "sfg_time_kernel": ([C.c_void_p, C.c_int, C.c_int, _fp], C.c_int),
    "sfg_time_kernel_flushed": ([C.c_void_p, C.c_int, C.c_int, C.c_size_t, C.POINTER(C.c_float)], C.c_int),
    "sfg_get_info": ([C.c_void_p, C.POINTER(Info)], C.c_int),
    "sfg_get_seismograms": ([C.c_void_p, _fp, C.c_size_t], C.c_int),
    "sfg_get_field": ([C.c_void_p, C.c_int, C.c_int, _fp, C.c_size_t], C.c_int),
    "sfg_get_numbering": ([C.c_void_p, _ip, _ip, _ip], C.c_int),
    "sfg_get_geometry": ([C.c_void_p, _dp, _dp, _dp, _ip], C.c_int),
    "sfg_check_finite": ([C.c_void_p], C.c_int),
    "sfg_set_model2d": ([C.c_void_p, _fp, _fp, _fp], C.c_int),
    "sfg_forward_checkpointed": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "sfg_adjoint_gradient": ([C.c_void_p, _fp, _fp, _fp, _fp], C.c_int),
    "sfg_set_adjoint_budget": ([C.c_void_p, C.c_size_t], C.c_int),
    "sfg_adjoint_buffers": ([C.c_void_p], C.c_int),
    "sfg_step_noalloc": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "sfg_predictor": ([C.c_void_p, C.c_int], C.c_int),
    "sfg_update_wavefields": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "sfg_corrector": ([C.c_void_p, C.c_int], C.c_int),
    "sfg_compute_seismograms": ([C.c_void_p, C.c_int], C.c_int),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libsfg.so and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libsfg is not built ({path}); run __graft_entry__.build()")
    lib = C.CDLL(path)
    for name, (args, res) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class SfgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


@dataclass
class Source:
    x: float
    z: float
    f0: float
    factor: float
    tshift: float = 0.0
    angle: float = 0.0
    stf: str = "ricker"
    shot: int = 0
    kind: str = "force"            # "force" or "moment_tensor"
    mxx: float = 0.0
    mzz: float = 0.0
    mxz: float = 0.0
    hdur: float = 0.0              # half duration of "gaussian_hdur" and "heaviside"


SOURCE_KIND = {"force": 0, "moment_tensor": 1}


def _arr(x, dtype):
    return np.ascontiguousarray(x, dtype=dtype)


class Simulation2D:
    """One 2D forward simulation on the GPU (a libsfg handle).

    ``mesh`` is any object with the attributes of ``sfg_mesh2d_desc``
    (nspec, npgeo, ngnod, coorg, knods, kmato, mat_medium, mat_rho, mat_vp,
    mat_vs, abs_ispec, abs_type, free_ispec, free_type), e.g. the meshes of
    ``specfempp_b200.meshgen``; or pass ``database=`` to read a database.bin.
    """

    def __init__(self, mesh=None, *, database: str | None = None, dt: float, nstep: int,
                 nshots: int = 1, nstep_between_samples: int = 1, elastic_wave: str = "psv",
                 point_rho=None, point_vp=None, point_vs=None, steps_per_graph: int = 0,
                 elements_per_block: int = 0, kernel_variant: int = 0,
                 store_acceleration: bool = False, start_time: float | None = None):
        self.lib = load_library()
        self._keep = []
        opt = Options(dt=dt, nstep=nstep, nshots=nshots, nstep_between_samples=nstep_between_samples,
                      steps_per_graph=steps_per_graph, elements_per_block=elements_per_block,
                      kernel_variant=kernel_variant, store_acceleration=int(store_acceleration),
                      has_start_time=int(start_time is not None),
                      start_time=float(start_time) if start_time is not None else 0.0)
        h = C.c_void_p()
        wave = 1 if elastic_wave.lower() == "sh" else 0
        if database is not None:
            rc = self.lib.sfg_create2d_from_database(database.encode(), wave, C.byref(opt), C.byref(h))
        else:
            d = self._desc(mesh, wave, point_rho, point_vp, point_vs)
            rc = self.lib.sfg_create2d(C.byref(d), C.byref(opt), C.byref(h))
        if rc != 0:
            raise SfgError(rc, self.lib.sfg_last_error(None).decode())
        self.h = h
        self.dt, self.nstep = dt, nstep
        self.ncomp = int(self.info().ncomp_elastic) or (1 if wave == 1 else 2)

    def _k(self, a):
        self._keep.append(a)
        return a

    def _desc(self, m, wave, prho, pvp, pvs):
        d = MeshDesc()
        d.nspec, d.npgeo, d.ngnod = int(m.nspec), int(m.npgeo), int(m.ngnod)
        d.coorg = self._k(_arr(m.coorg, np.float64)).ctypes.data_as(_dp)
        d.knods = self._k(_arr(m.knods, np.int32)).ctypes.data_as(_ip)
        d.kmato = self._k(_arr(m.kmato, np.int32)).ctypes.data_as(_ip)
        d.numat = len(m.mat_rho)
        d.mat_medium = self._k(_arr(m.mat_medium, np.int32)).ctypes.data_as(_ip)
        d.mat_rho = self._k(_arr(m.mat_rho, np.float64)).ctypes.data_as(_dp)
        d.mat_vp = self._k(_arr(m.mat_vp, np.float64)).ctypes.data_as(_dp)
        d.mat_vs = self._k(_arr(m.mat_vs, np.float64)).ctypes.data_as(_dp)
        for name, a in (("point_rho", prho), ("point_vp", pvp), ("point_vs", pvs)):
            if a is not None:
                setattr(d, name, self._k(_arr(a, np.float32)).ctypes.data_as(_fp))
        d.nabs = len(m.abs_ispec)
        d.abs_ispec = self._k(_arr(m.abs_ispec, np.int32)).ctypes.data_as(_ip)
        d.abs_type = self._k(_arr(m.abs_type, np.int32)).ctypes.data_as(_ip)
        d.nfree = len(m.free_ispec)
        d.free_ispec = self._k(_arr(m.free_ispec, np.int32)).ctypes.data_as(_ip)
        d.free_type = self._k(_arr(m.free_type, np.int32)).ctypes.data_as(_ip)
        d.elastic_wave = wave
        cos = getattr(m, "mat_cosserat", None)
        if cos is not None:
            cos = _arr(cos, np.float64).reshape(len(m.mat_rho), 8)
            d.mat_cosserat = self._k(np.ascontiguousarray(cos)).ctypes.data_as(_dp)
        aniso = getattr(m, "mat_aniso", None)
        if aniso is not None:
            aniso = _arr(aniso, np.float64).reshape(len(m.mat_rho), 6)
            d.mat_aniso = self._k(np.ascontiguousarray(aniso)).ctypes.data_as(_dp)
        poro = getattr(m, "mat_poro", None)
        if poro is not None:
            poro = _arr(poro, np.float64).reshape(len(m.mat_rho), 13)
            d.mat_poro = self._k(np.ascontiguousarray(poro)).ctypes.data_as(_dp)
        adj = getattr(m, "adjacency", None)
        if adj is None:
            adj = getattr(m, "extra", {}).get("adjacency")
        if adj is not None and len(adj):
            adj = _arr(adj, np.int32).reshape(-1, 4)
            d.nadj = len(adj)
            d.adjacency = self._k(np.ascontiguousarray(adj)).ctypes.data_as(_ip)
        return d

    def _check(self, rc):
        if rc != 0:
            raise SfgError(rc, self.lib.sfg_last_error(self.h).decode())

    def set_sources(self, sources):
        arr = (Source2D * len(sources))()
        for i, s in enumerate(sources):
            arr[i] = Source2D(x=s.x, z=s.z, shot=getattr(s, "shot", 0), stf=STF[getattr(s, "stf", "ricker")],
                              f0=s.f0, factor=s.factor, tshift=getattr(s, "tshift", 0.0),
                              angle=getattr(s, "angle", 0.0),
                              kind=SOURCE_KIND[getattr(s, "kind", "force")],
                              mxx=getattr(s, "mxx", 0.0), mzz=getattr(s, "mzz", 0.0),
                              mxz=getattr(s, "mxz", 0.0), hdur=getattr(s, "hdur", 0.0))
        self._check(self.lib.sfg_set_sources(self.h, len(sources), arr))

    def set_stf_table(self, table):
        t = _arr(table, np.float32)
        self._check(self.lib.sfg_set_stf_table(self.h, t.ctypes.data_as(_fp), t.shape[0], t.shape[1]))

    def set_receivers(self, x, z, angle=0.0, types=("displacement",)):
        x = _arr(x, np.float64)
        z = _arr(z, np.float64)
        ty = _arr([SEIS[t] for t in types], np.int32)
        self._check(self.lib.sfg_set_receivers(self.h, len(x), x.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                                               float(angle), len(ty), ty.ctypes.data_as(_ip)))

    def initialize(self):
        self._check(self.lib.sfg_initialize(self.h))

    def step(self):
        self._check(self.lib.sfg_step(self.h))

    def run(self, nsteps):
        self._check(self.lib.sfg_run(self.h, int(nsteps)))

    def run_timed(self, nsteps) -> float:
        ms = C.c_float()
        self._check(self.lib.sfg_run_timed(self.h, int(nsteps), C.byref(ms)))
        return ms.value

    def run_timed_flushed(self, nsteps, flush_bytes=256 << 20) -> float:
        ms = C.c_float()
        self._check(self.lib.sfg_run_timed_flushed(self.h, int(nsteps), int(flush_bytes), C.byref(ms)))
        return ms.value

    def step_io(self, stf_row=None, seis_row=None):
        """One step with host buffers (contiguous float32 numpy arrays, ideally
        pinned): the sources' time-function values of the step in, the step's
        seismogram row out."""
        sp = stf_row.ctypes.data if stf_row is not None else None
        op = seis_row.ctypes.data if seis_row is not None else None
        rc = self.lib.sfg_step_io(self.h, sp, op)
        if rc:
            self._check(rc)

    def time_kernel(self, which: int, iters: int, flush_bytes: int = 0) -> float:
        """Average device ms of one launch of a kernel family (sfg_time_kernel);
        with flush_bytes > 0 the L2 is flushed before every launch."""
        ms = C.c_float()
        self._check(self.lib.sfg_time_kernel_flushed(self.h, int(which), int(iters), int(flush_bytes),
                                                     C.byref(ms)))
        return ms.value

    def synchronize(self):
        self._check(self.lib.sfg_synchronize(self.h))

    def reset(self):
        self._check(self.lib.sfg_reset_fields(self.h))

    def info(self) -> Info:
        inf = Info()
        self._check(self.lib.sfg_get_info(self.h, C.byref(inf)))
        return inf

    def seismograms(self) -> np.ndarray:
        """[nshots, nsig, ntypes, nrec, 2] float32."""
        i = self.info()
        out = np.zeros((i.nshots, i.nsig, i.ntypes, i.nrec, 2), np.float32)
        self._check(self.lib.sfg_get_seismograms(self.h, out.ctypes.data_as(_fp), out.size))
        return out

    def field(self, medium: str, which: str = "displacement") -> np.ndarray:
        """Field of one medium in the handle's point numbering: elastic [nglob, ncomp]
        (with nshots > 1: [nshots, nglob, ncomp]), acoustic [nglob]."""
        i = self.info()
        med = SFG_MEDIUM_ELASTIC if medium == "elastic" else SFG_MEDIUM_ACOUSTIC
        n = i.nglob_elastic if med == SFG_MEDIUM_ELASTIC else i.nglob_acoustic
        nc = self.ncomp if med == SFG_MEDIUM_ELASTIC else 1
        out = np.zeros(i.nshots * n * nc, np.float32)
        self._check(self.lib.sfg_get_field(self.h, med, FIELD[which], out.ctypes.data_as(_fp), out.size))
        if med == SFG_MEDIUM_ACOUSTIC:
            return out if i.nshots == 1 else out.reshape(i.nshots, n)
        return out.reshape(n, nc) if i.nshots == 1 else out.reshape(i.nshots, n, nc)

    def numbering(self):
        i = self.info()
        ib = np.zeros(i.nspec * 25, np.int32)
        g2e = np.zeros(i.nglob, np.int32)
        g2a = np.zeros(i.nglob, np.int32)
        self._check(self.lib.sfg_get_numbering(self.h, ib.ctypes.data_as(_ip), g2e.ctypes.data_as(_ip),
                                               g2a.ctypes.data_as(_ip)))
        return ib.reshape(i.nspec, 25), g2e, g2a

    def geometry(self):
        """(x, z, |J|) of every element GLL point [nspec, 25] (database element
        order, FP64) and the medium of every element (0 acoustic, 1 elastic)."""
        n = self.info().nspec
        x, z, jac = (np.zeros((n, 25)) for _ in range(3))
        med = np.zeros(n, np.int32)
        self._check(self.lib.sfg_get_geometry(self.h, x.ctypes.data_as(_dp), z.ctypes.data_as(_dp),
                                              jac.ctypes.data_as(_dp), med.ctypes.data_as(_ip)))
        return x, z, jac, med

    def check_finite(self) -> bool:
        rc = self.lib.sfg_check_finite(self.h)
        if rc not in (0, -6):
            self._check(rc)
        return rc == 0

    # ---- adjoint -------------------------------------------------------
    def set_model(self, rho, kappa, mu):
        """Per-GLL-point model [nspec, 25] (database element order)."""
        r, k, m = (_arr(x, np.float32) for x in (rho, kappa, mu))
        self._check(self.lib.sfg_set_model2d(self.h, r.ctypes.data_as(_fp), k.ctypes.data_as(_fp),
                                             m.ctypes.data_as(_fp)))

    def forward_checkpointed(self, nsteps, interval):
        self._check(self.lib.sfg_forward_checkpointed(self.h, int(nsteps), int(interval)))
        return self.seismograms()[0, :nsteps, 0]

    def set_adjoint_budget(self, nbytes: int):
        """Device bytes for the adjoint's segment buffers (0: 75% of the free
        memory); the forward run keeps as many recorded segments as they hold."""
        self._check(self.lib.sfg_set_adjoint_budget(self.h, int(nbytes)))

    def adjoint_buffers(self) -> int:
        """Segment buffers of the last checkpointed forward run (0 before)."""
        return int(self.lib.sfg_adjoint_buffers(self.h))

    def adjoint_gradient(self, seis_grad):
        """dL/d(rho, kappa, mu) per GLL point [nspec, 25] given dL/dseis [nsteps, nrec, 2]."""
        i = self.info()
        g = _arr(seis_grad, np.float32)
        out = [np.zeros((i.nspec, 25), np.float32) for _ in range(3)]
        self._check(self.lib.sfg_adjoint_gradient(self.h, g.ctypes.data_as(_fp),
                                                  *[o.ctypes.data_as(_fp) for o in out]))
        return tuple(out)

    def close(self):
        if getattr(self, "h", None):
            self.lib.sfg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
