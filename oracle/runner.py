"""ctypes front-end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
may import this module.  It loads ``oracle/_build/liboracle.so`` (built by
``oracle/Makefile``), turns a mesh plus source/receiver description into the
plain arrays of ``OracleInput2D`` and returns seismograms as numpy arrays.

The start time follows ``src/io/sources/dim2/read_sources.cpp:142-172``: t0 is
the minimum of the sources' ``-1.2/f0 + tshift`` and each source's tshift is
replaced by ``t0_source - t0``.  Seismogram times are
``isig * dt * nstep_between_samples + t0``
(``core/specfem/assembly/receivers/dim2/impl/seismogram_iterator.hpp:38``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

from .database2d import Mesh2D, read_database

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
# the same sources built for x86-64-v3 (AVX2, hardware FMA): the same bits
LIB_PATH_V3 = os.path.join(HERE, "_build", "liboracle_v3.so")
_V3_FLAGS = {"avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "abm", "movbe", "xsave"}


def cpu_has_x86_64_v3() -> bool:
    """Whether the host CPU lists the x86-64-v3 instruction sets (Linux)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return _V3_FLAGS <= set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return False

SEIS_TYPES = {"displacement": 0, "velocity": 1, "acceleration": 2, "pressure": 3,
              "rotation": 4, "intrinsic_rotation": 5, "curl": 6}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OracleInput2D(C.Structure):
    _fields_ = [
        ("nspec", C.c_int), ("npgeo", C.c_int), ("ngnod", C.c_int),
        ("coorg", _dp), ("knods", _ip), ("medium", _ip),
        ("rho", _dp), ("vp", _dp), ("vs", _dp),
        ("elastic_sh", C.c_int),
        ("nabs", C.c_int), ("abs_ispec", _ip), ("abs_type", _ip),
        ("nfree", C.c_int), ("free_ispec", _ip), ("free_type", _ip),
        ("nsrc", C.c_int), ("src_x", _dp), ("src_z", _dp), ("src_angle", _dp),
        ("src_f0", _dp), ("src_factor", _dp), ("src_tshift", _dp),
        ("stf_table", _dp), ("t0", C.c_double),
        ("nrec", C.c_int), ("rec_x", _dp), ("rec_z", _dp), ("rec_angle", C.c_double),
        ("ntypes", C.c_int), ("seis_types", _ip),
        ("dt", C.c_double), ("nstep", C.c_int), ("nstep_between_samples", C.c_int),
        ("setup_in_run_precision", C.c_int),
        ("src_kind", _ip), ("src_mxx", _dp), ("src_mzz", _dp), ("src_mxz", _dp),
        ("aniso", _dp), ("cosserat", _dp),
        ("nadj", C.c_int), ("adjacency", _ip), ("poro", _dp),
        ("device_order", C.c_int)]


class OracleOutput2D(C.Structure):
    _fields_ = [
        ("seismograms", _dp), ("final_u_elastic", _dp), ("final_u_acoustic", _dp),
        ("ibool", _ip), ("nglob", C.c_int), ("loop_seconds", C.c_double),
        ("error", C.c_char * 256),
    ]


_lib = None


def build() -> str:
    """Compile the oracle shared libraries with their Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib_path() -> str:
    """The library this host runs: the x86-64-v3 build where the CPU has its
    instructions, else the baseline build."""
    return LIB_PATH_V3 if cpu_has_x86_64_v3() else LIB_PATH


def lib():
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            build()
        _lib = C.CDLL(path)
        for name in ("oracle2d_run_f32", "oracle2d_run_f64"):
            fn = getattr(_lib, name)
            fn.argtypes = [C.POINTER(OracleInput2D), C.POINTER(OracleOutput2D), C.c_int]
            fn.restype = C.c_int
        _lib.oracle2d_count_nglob.argtypes = [C.POINTER(OracleInput2D)]
        _lib.oracle2d_count_nglob.restype = C.c_int
        _lib.oracle_gll.argtypes = [_dp, _dp, _dp]
        _lib.oracle_legendre.argtypes = [C.c_double, C.c_int]
        _lib.oracle_legendre.restype = C.c_double
        _lib.oracle_stress_psv.argtypes = [C.c_double, C.c_double, _dp, _dp]
    return _lib


@dataclass
class Source:
    x: float
    z: float
    f0: float
    factor: float
    tshift: float = 0.0
    angle: float = 0.0
    stf: str = "ricker"          # ricker, dirac, gaussian, dgaussian, gaussian_hdur, heaviside
    kind: str = "force"          # "force" or "moment_tensor"
    mxx: float = 0.0
    mzz: float = 0.0
    mxz: float = 0.0
    hdur: float = 0.0            # half duration (gaussian_hdur, heaviside)


@dataclass
class Case2D:
    mesh: Mesh2D
    sources: list
    rec_x: np.ndarray
    rec_z: np.ndarray
    dt: float
    nstep: int
    seis_types: list = field(default_factory=lambda: ["displacement"])
    nstep_between_samples: int = 1
    rec_angle: float = 0.0
    elastic_sh: bool = False
    point_rho: np.ndarray | None = None   # optional per-GLL-point models [nspec, 25]
    point_vp: np.ndarray | None = None
    point_vs: np.ndarray | None = None
    stf_table: np.ndarray | None = None    # optional [nstep, nsrc]
    stations: list = field(default_factory=list)
    setup_in_run_precision: bool = False   # True: reference-faithful FP32 setup geometry
    device_order: bool = False             # True: FMA contractions as the CUDA kernels evaluate them
    start_time: float | None = None        # the configuration's t0 (sources keep their tshift)


def _src_start(s, dt):
    """Start time and evaluation parameter of one source, FP32: -1.2/f0 +
    tshift for ricker / dirac / dgaussian (ricker.cpp:18-21, dgaussian.cpp:17-20),
    -2/f0 + tshift for gaussian (gaussian.cpp:17-21, the 2D factor of
    core/specfem/source/source.tpp:17-62), and for gaussian_hdur / heaviside
    hdur raised to 5 dt, start -2 hdur + tshift, evaluated with hdur / 1.628
    (gaussianhdur.cpp:17-37, heaviside.cpp:15-34)."""
    f32 = np.float32
    if s.stf in ("gaussian_hdur", "heaviside"):
        h = f32(s.hdur)
        if h < f32(5.0) * f32(dt if dt is not None else 0.0):
            h = f32(5.0) * f32(dt)
        return f32(-f32(2.0) * h + f32(s.tshift)), f32(h / f32(1.628))
    k = f32(2.0) if s.stf == "gaussian" else f32(1.2)
    return f32(-k * (f32(1.0) / f32(s.f0)) + f32(s.tshift)), f32(s.f0)


def start_time(sources, dt=None) -> tuple[float, list]:
    """t0 and effective tshifts (read_sources.cpp:142-172), in FP32 like the reference."""
    t0s = [_src_start(s, dt)[0] for s in sources]
    t0 = min(t0s)
    return float(t0), [float(t - t0) for t in t0s]


def point_models(case: Case2D):
    m = case.mesh
    if case.point_rho is not None:
        return (np.ascontiguousarray(case.point_rho, np.float64),
                np.ascontiguousarray(case.point_vp, np.float64),
                np.ascontiguousarray(case.point_vs, np.float64))
    rho = np.repeat(m.mat_rho[m.kmato][:, None], 25, axis=1)
    vp = np.repeat(m.mat_vp[m.kmato][:, None], 25, axis=1)
    vs = np.repeat(m.mat_vs[m.kmato][:, None], 25, axis=1)
    return rho, vp, vs


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def aniso_points(case):
    """[nspec, 25, 6] anisotropic constants when the mesh has an anisotropic
    material (isotropic elements as c11 = c33 = lambda + 2 mu, c13 = lambda,
    c55 = mu, c15 = c35 = 0), else None."""
    m = case.mesh
    ma = getattr(m, "mat_aniso", None)
    if ma is None or not np.isfinite(ma).any():
        return None
    rho, vp, vs = point_models(case)
    mu = rho * vs * vs
    l2m = rho * vp * vp
    iso = np.stack([l2m, l2m - 2 * mu, 0 * mu, l2m, 0 * mu, mu], -1)      # [nspec, 25, 6]
    per = ma[m.kmato]                                                    # [nspec, 6]
    out = np.where(np.isfinite(per)[:, None, :], per[:, None, :], iso)
    return np.ascontiguousarray(out)


def nonconforming_records(m):
    """The mesh's nonconforming adjacency records [n][4] (element, neighbour,
    3, edge type), 0-based; the strongly conforming ones are implied by the
    shared control nodes."""
    adj = getattr(m, "adjacency", None)
    if adj is None:
        adj = getattr(m, "extra", {}).get("adjacency")
    if adj is None or len(adj) == 0:
        return np.zeros((0, 4), np.int32)
    adj = np.asarray(adj, np.int32).reshape(-1, 4)
    return np.ascontiguousarray(adj[adj[:, 2] == 3])


def poro_points(case):
    """[nspec, 25, 13] poroelastic constants (rho_s, rho_f, phi, tortuosity,
    kxx, kxz, kzz, kappa_s, kappa_f, kappa_fr, eta_f, mu_fr, Q_mu) when the mesh
    has poroelastic materials, else None; every elastic element must then be
    poroelastic."""
    m = case.mesh
    mp = getattr(m, "mat_poro", None)
    if mp is None or not np.isfinite(mp).any():
        return None
    per = np.asarray(mp)[m.kmato]
    elastic = np.asarray(m.mat_medium)[m.kmato] == 1
    if not np.all(np.isfinite(per[elastic])):
        raise ValueError("a mesh with poroelastic materials must be poroelastic in every elastic element")
    per = np.where(np.isfinite(per), per, 0.0)
    return np.ascontiguousarray(np.repeat(per[:, None, :], 25, axis=1))


def cosserat_points(case):
    """[nspec, 25, 8] Cosserat constants (rho, kappa, mu, nu, j, lambda_c,
    mu_c, nu_c) when the mesh has Cosserat materials, else None; every elastic
    element must then be Cosserat."""
    m = case.mesh
    mc = getattr(m, "mat_cosserat", None)
    if mc is None or not np.isfinite(mc).any():
        return None
    per = np.asarray(mc)[m.kmato]                                     # [nspec, 8]
    elastic = np.asarray(m.mat_medium)[m.kmato] == 1
    if not np.all(np.isfinite(per[elastic])):
        raise ValueError("a mesh with Cosserat materials must be Cosserat in every elastic element")
    per = np.where(np.isfinite(per), per, 0.0)
    return np.ascontiguousarray(np.repeat(per[:, None, :], 25, axis=1))


def _make_input(case: Case2D, keep: list):
    """OracleInput2D of a case (arrays kept alive in `keep`); also returns the
    seismogram type codes and the sampling interval."""
    m = case.mesh

    def arr(x, dt):
        a = np.ascontiguousarray(x, dtype=dt)
        keep.append(a)
        return a

    rho, vp, vs = point_models(case)
    srcs = [effective_f0(s, case.dt) for s in case.sources]
    t0, tsh = start_time(srcs, case.dt)
    stf_table = case.stf_table
    if case.start_time is not None:
        # read_sources.cpp:155-161: the given start, each source's own tshift
        t0, tsh = float(np.float32(case.start_time)), [float(np.float32(s.tshift)) for s in srcs]
        if stf_table is None:
            stf_table = stf_tables(case.sources, case.dt, case.nstep, start=case.start_time)
    if stf_table is None and any(s.stf != "ricker" for s in srcs):
        stf_table = stf_tables(case.sources, case.dt, case.nstep)
    inp = OracleInput2D()
    inp.nspec, inp.npgeo, inp.ngnod = m.nspec, m.npgeo, m.ngnod
    inp.coorg = _ptr(arr(m.coorg, np.float64), _dp)
    inp.knods = _ptr(arr(m.knods, np.int32), _ip)
    inp.medium = _ptr(arr(m.mat_medium[m.kmato], np.int32), _ip)
    inp.rho, inp.vp, inp.vs = (_ptr(arr(a, np.float64), _dp) for a in (rho, vp, vs))
    inp.elastic_sh = int(case.elastic_sh)
    inp.nabs = len(m.abs_ispec)
    inp.abs_ispec = _ptr(arr(m.abs_ispec, np.int32), _ip)
    inp.abs_type = _ptr(arr(m.abs_type, np.int32), _ip)
    inp.nfree = len(m.free_ispec)
    inp.free_ispec = _ptr(arr(m.free_ispec, np.int32), _ip)
    inp.free_type = _ptr(arr(m.free_type, np.int32), _ip)
    inp.nsrc = len(srcs)
    inp.src_x = _ptr(arr([s.x for s in srcs], np.float64), _dp)
    inp.src_z = _ptr(arr([s.z for s in srcs], np.float64), _dp)
    inp.src_angle = _ptr(arr([s.angle for s in srcs], np.float64), _dp)
    inp.src_f0 = _ptr(arr([s.f0 for s in srcs], np.float64), _dp)
    inp.src_factor = _ptr(arr([s.factor for s in srcs], np.float64), _dp)
    inp.src_tshift = _ptr(arr(tsh, np.float64), _dp)
    inp.stf_table = _ptr(arr(stf_table, np.float64), _dp) if stf_table is not None else None
    inp.t0 = t0
    inp.nrec = len(case.rec_x)
    inp.rec_x = _ptr(arr(case.rec_x, np.float64), _dp)
    inp.rec_z = _ptr(arr(case.rec_z, np.float64), _dp)
    inp.rec_angle = case.rec_angle
    types = [SEIS_TYPES[t] for t in case.seis_types]
    inp.ntypes = len(types)
    inp.seis_types = _ptr(arr(types, np.int32), _ip)
    inp.dt, inp.nstep = case.dt, case.nstep
    nsb = max(1, case.nstep_between_samples)
    inp.nstep_between_samples = nsb
    inp.setup_in_run_precision = int(case.setup_in_run_precision)
    inp.device_order = int(case.device_order)
    inp.src_kind = _ptr(arr([1 if getattr(s, "kind", "force") == "moment_tensor" else 0 for s in srcs],
                            np.int32), _ip)
    inp.src_mxx = _ptr(arr([getattr(s, "mxx", 0.0) for s in srcs], np.float64), _dp)
    inp.src_mzz = _ptr(arr([getattr(s, "mzz", 0.0) for s in srcs], np.float64), _dp)
    inp.src_mxz = _ptr(arr([getattr(s, "mxz", 0.0) for s in srcs], np.float64), _dp)
    aniso = aniso_points(case)
    inp.aniso = _ptr(arr(aniso, np.float64), _dp) if aniso is not None else None
    cos = cosserat_points(case)
    inp.cosserat = _ptr(arr(cos, np.float64), _dp) if cos is not None else None
    poro = poro_points(case)
    inp.poro = _ptr(arr(poro, np.float64), _dp) if poro is not None else None
    adj = nonconforming_records(m)
    inp.nadj = len(adj)
    inp.adjacency = _ptr(arr(adj, np.int32), _ip) if len(adj) else None
    return inp, types, nsb


def run(case: Case2D, precision: str = "f32", nthreads: int = 1, want_final: bool = False):
    """Run the oracle; returns dict with 'seis' [nsig, ntypes, nrec, 2], 't0', 'times'."""
    m = case.mesh
    L = lib()
    keep = []
    inp, types, nsb = _make_input(case, keep)
    t0 = inp.t0
    poro, cos = poro_points(case), cosserat_points(case)
    nsig = (case.nstep + nsb - 1) // nsb
    seis = np.zeros((nsig, len(types), len(case.rec_x), 2))
    out = OracleOutput2D()
    out.seismograms = _ptr(seis, _dp)
    final = None
    if want_final:
        nglob = L.oracle2d_count_nglob(C.byref(inp))
        nce = 4 if poro is not None else 3 if cos is not None else 1 if case.elastic_sh else 2
        final = {"elastic": np.zeros((nglob, nce)),
                 "acoustic": np.zeros(nglob),
                 "ibool": np.zeros((m.nspec, 25), np.int32)}
        out.final_u_elastic = _ptr(final["elastic"], _dp)
        out.final_u_acoustic = _ptr(final["acoustic"], _dp)
        out.ibool = _ptr(final["ibool"], _ip)
    fn = L.oracle2d_run_f32 if precision == "f32" else L.oracle2d_run_f64
    rc = fn(C.byref(inp), C.byref(out), int(nthreads))
    if rc != 0:
        raise RuntimeError(out.error.decode())
    times = np.arange(nsig) * (case.dt * nsb) + t0
    return {"seis": seis, "t0": t0, "times": times, "final": final, "nglob": out.nglob,
            "loop_seconds": out.loop_seconds}


def adjoint_compat(case: Case2D, adj, quirk: bool = False, reconstruct: bool = True):
    """The reference's combined adjoint simulation and Frechet kernels (FP64)
    of an isotropic elastic P-SV case: adjoint sources adj [nstep][nrec][2]
    at the receivers; kernels rho, mu, kappa [nspec, 25] (mesh element order)
    as the reference accumulates them (kappa with respect to kappa2D =
    lambda + mu), and the quadrature weight w_x w_z |J| of every point.
    quirk: the backward field's derivatives include the adjoint field's, as
    the reference's two-field gradient computes them; reconstruct: the
    reference's reverse-time backward field (else the forward snapshots)."""
    L = lib()
    keep = []
    inp, _, _ = _make_input(case, keep)
    n = case.mesh.nspec * 25
    out = {k: np.zeros((case.mesh.nspec, 25)) for k in ("rho", "mu", "kappa", "weight")}
    a = np.ascontiguousarray(adj, np.float64)
    if a.shape != (case.nstep, len(case.rec_x), 2):
        raise ValueError("adjoint sources must be [nstep, nrec, 2]")
    err = C.create_string_buffer(256)
    fn = L.oracle2d_adjoint_compat_f64
    fn.argtypes = [C.POINTER(OracleInput2D), _dp, C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_char_p, C.c_int]
    fn.restype = C.c_int
    rc = fn(C.byref(inp), _ptr(a, _dp), int(quirk), int(reconstruct), _ptr(out["rho"], _dp), _ptr(out["mu"], _dp),
            _ptr(out["kappa"], _dp), _ptr(out["weight"], _dp), err, 256)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    assert out["rho"].size == n
    return out


# ------------------------------------------------ reference fixtures ---

def read_stations(path):
    names, xs, zs = [], [], []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) < 4:
                continue
            names.append((p[1], p[0]))
            xs.append(float(p[2]))
            zs.append(float(p[3]))
    return names, np.asarray(xs), np.asarray(zs)


def read_sources_yaml(path):
    import yaml
    with open(path) as f:
        d = yaml.safe_load(f)
    out = []
    for s in d["sources"]:
        if "force" in s:
            fs, kind_src = s["force"], "force"
        elif "moment-tensor" in s:
            fs, kind_src = s["moment-tensor"], "moment_tensor"
        else:
            raise ValueError("only force and moment-tensor sources are on this path")
        rk = kind = None
        for key, k in (("Ricker", "ricker"), ("Dirac", "dirac"), ("dGaussian", "dgaussian"),
                       ("Heaviside", "heaviside")):
            if key in fs:
                rk, kind = fs[key], k
        if "Gaussian" in fs:
            rk = fs["Gaussian"]
            kind = "gaussian_hdur" if "hdur" in rk else "gaussian"
        if rk is None:
            raise ValueError("time function not on this path")
        out.append(Source(x=float(fs["x"]), z=float(fs["z"]), f0=float(rk.get("f0", 0.0)),
                          factor=float(rk["factor"]), tshift=float(rk.get("tshift", 0.0)),
                          angle=float(fs.get("angle", 0.0)), stf=kind, kind=kind_src,
                          mxx=float(fs.get("Mxx", 0.0)), mzz=float(fs.get("Mzz", 0.0)),
                          mxz=float(fs.get("Mxz", 0.0)), hdur=float(rk.get("hdur", 0.0))))
    return out


def stf_tables(sources, dt, nstep, start=None):
    """FP32 source-time-function table [nstep, nsrc]
    (core/specfem/source_time_functions/impl/time_functions.hpp), a = pi^2 f0^2:
    ricker factor (1 - 2 a t^2) exp(-a t^2); dirac (f0 = 1/(10 dt)) and
    gaussian factor (-exp(-a t^2) / (2a)); dgaussian factor t exp(-a t^2);
    gaussian_hdur factor exp(-t^2/h^2) / (sqrt(pi) h); heaviside factor
    (1 + erf(t/h)) / 2; t = t0 + i dt - tshift.
    """
    import math
    f32 = np.float32
    srcs = [effective_f0(s, dt) for s in sources]
    t0, tsh = start_time(srcs, dt)
    if start is not None:
        t0, tsh = float(f32(start)), [float(f32(s.tshift)) for s in srcs]
    i = np.arange(nstep, dtype=f32)
    tab = np.zeros((nstep, len(srcs)), np.float32)
    pi = f32(np.pi)
    for k, s in enumerate(srcs):
        t = f32(t0) + i * f32(dt) - f32(tsh[k])
        fac = f32(s.factor)
        p = _src_start(s, dt)[1]
        if s.stf == "heaviside":
            e = np.array([math.erf(float(v)) for v in t / p], dtype=f32)
            tab[:, k] = fac * (f32(0.5) * (f32(1.0) + e))
            continue
        if s.stf == "gaussian_hdur":
            tab[:, k] = fac * (np.exp(-(f32(1.0) / (p * p)) * t * t) / (f32(math.sqrt(math.pi)) * p))
            continue
        a = pi * pi * p * p
        if s.stf in ("dirac", "gaussian"):
            tab[:, k] = fac * (f32(-1.0) * np.exp(-a * t * t) / (f32(2.0) * a))
        elif s.stf == "dgaussian":
            tab[:, k] = fac * (t * np.exp(-a * t * t))
        else:
            tab[:, k] = fac * ((f32(1.0) - f32(2.0) * a * t * t) * np.exp(-a * t * t))
    return tab


def effective_f0(s, dt):
    """Dirac sources use f0 = 1/(10 dt) (dirac.cpp:25)."""
    if s.stf == "dirac":
        from dataclasses import replace
        return replace(s, f0=float(np.float32(1.0) / (np.float32(10.0) * np.float32(dt))))
    return s


def load_fixture(fixture_dir, types=("displacement",)):
    """Load a reference Newmark fixture directory into a Case2D."""
    import yaml
    with open(os.path.join(fixture_dir, "specfem_config.yaml")) as f:
        cfg = yaml.safe_load(f)["parameters"]
    ts = cfg["simulation-setup"]["solver"]["time-marching"]["time-scheme"]
    rc = cfg["receivers"]
    mesh = read_database(os.path.join(fixture_dir, "database.bin"))

    def local(path, default):
        # the configuration's paths are relative to the test tree: a file of
        # this fixture, else of the sibling fixture it names
        path = str(path or default)
        own = os.path.join(fixture_dir, os.path.basename(path))
        if os.path.exists(own):
            return own
        return os.path.join(os.path.dirname(os.path.abspath(fixture_dir)),
                            os.path.basename(os.path.dirname(path)), os.path.basename(path))

    names, rx, rz = read_stations(local(rc.get("stations"), "STATIONS"))
    src = read_sources_yaml(local(cfg.get("sources"), "sources.yaml"))   # sources.yaml or source.yaml
    sh = str(cfg["simulation-setup"].get("elastic-wave", "P_SV")).upper() == "SH"
    return Case2D(mesh=mesh, sources=src, rec_x=rx, rec_z=rz, dt=float(ts["dt"]),
                  nstep=int(ts["nstep"]), seis_types=list(types),
                  nstep_between_samples=int(rc.get("nstep_between_samples", 1)),
                  rec_angle=float(rc.get("angle", 0.0)), stations=names, elastic_sh=sh)


def read_trace(path):
    a = np.loadtxt(path)
    return a[:, 0], a[:, 1]


def reference_metric(computed, fixture_dir, stations, kind="semd", comps=("BXX", "BXZ")):
    """Per-station sum|d| / sum|ref| as in newmark_tests.cpp:331-373.

    ``computed`` is [nsig, nrec, ncomp] for one seismogram type.
    """
    errs = []
    for r, (net, sta) in enumerate(stations):
        err = norm = 0.0
        for c, comp in enumerate(comps):
            t, v = read_trace(os.path.join(fixture_dir, "traces", f"{net}.{sta}.S2.{comp}.{kind}"))
            n = min(len(v), computed.shape[0])
            err += np.abs(computed[:n, r, c] - v[:n]).sum()
            norm += np.abs(v[:n]).sum()
        errs.append(err / norm if norm > 0 else float("nan"))
    return np.asarray(errs)
