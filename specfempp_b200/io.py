"""Reference-format inputs and outputs of the 2D forward run.

* ``read_config``: the subset of a SPECFEM++ ``specfem_config.yaml`` that a
  forward Newmark run needs (src/parameter_parser/setup.cpp and the
  ``parameters`` keys of the reference's example configurations);
* ``read_stations``: a 2D STATIONS file (station, network, x, z, ...);
* ``read_sources``: a ``sources.yaml`` with force and moment-tensor sources,
  Ricker or Dirac time functions (src/io/sources/dim2/read_sources.cpp);
* ``write_seismograms_ascii``: one two-column ``time value`` file per station,
  component and seismogram type, named ``NET.STA.S2.<channel>.<ext>`` like the
  reference's writer (src/io/seismogram/writer.cpp:8-141);
* ``write_kernels``: Frechet kernels in the folder layout of the reference's
  kernel writer (include/io/kernel/writer.tpp, include/io/impl/medium_writer.tpp);
* ``WavefieldWriter``: wavefield snapshots in the layout of the reference's
  wavefield writer (include/io/wavefield/writer.tpp);
both through the reference's ASCII (``<name>.txt`` + ``<name>.meta``) or NPY
(``<name>.npy``) output libraries (include/io/ASCII, include/io/NPY), read
back by ``read_dataset``.
"""
from __future__ import annotations

import os
import shutil
from dataclasses import dataclass, field

import numpy as np

EXT = {"displacement": "semd", "velocity": "semv", "acceleration": "sema", "pressure": "semp",
       "rotation": "semr", "intrinsic_rotation": "semir", "curl": "semc"}


@dataclass
class ForwardConfig:
    dt: float
    nstep: int
    elastic_wave: str                 # "psv" or "sh"
    database: str                     # path of database.bin
    sources: object                   # path of sources.yaml, or the sources node itself
    stations: object                  # path of STATIONS, or the YAML list of stations
    angle: float = 0.0
    seismogram_types: list = field(default_factory=lambda: ["displacement"])
    nstep_between_samples: int = 1
    output_directory: str = "."
    output_format: str = "ascii"
    # wavefield writer (simulation-mode/forward/writer/wavefield): folder,
    # library, snapshot every `wavefield_interval` steps (0: none) and at the
    # last step when `wavefield_last_step` (src/parameter_parser/writer/wavefield.cpp)
    wavefield_directory: str | None = None
    wavefield_format: str = "ascii"
    wavefield_interval: int = 0
    wavefield_last_step: bool = True
    start_time: float | None = None   # time-scheme t0 (sources keep their tshift)


def _resolve(path, roots):
    if os.path.isabs(path):
        return path
    for r in roots:
        cand = os.path.join(r, path)
        if os.path.exists(cand):
            return cand
    return os.path.join(roots[0], path)


def read_config(path: str, root: str | None = None) -> ForwardConfig:
    """Parse a reference ``specfem_config.yaml``; relative paths are looked up
    under ``root`` (the directory the reference runs from), the config's own
    directory and the working directory, in that order."""
    import yaml
    with open(path) as f:
        cfg = yaml.safe_load(f)["parameters"]
    setup = cfg["simulation-setup"]
    ts = setup["solver"]["time-marching"]["time-scheme"]
    if str(ts.get("type", "Newmark")).lower() != "newmark":
        raise ValueError("only the Newmark time scheme is on this path")
    tos = str(setup["solver"]["time-marching"].get("type-of-simulation", "forward")).lower()
    if tos != "forward":
        raise ValueError("only forward simulations are driven from a configuration file")
    wave = str(setup.get("elastic-wave", "P_SV")).replace("-", "_").upper()
    rc = cfg["receivers"]
    roots = [r for r in (root, os.path.dirname(os.path.abspath(path)), os.getcwd()) if r]
    out_dir, out_fmt = ".", "ascii"
    mode = setup.get("simulation-mode", {}).get("forward", {}) or {}
    seis_w = (mode.get("writer", {}) or {}).get("seismogram", {}) or {}
    if seis_w:
        out_dir = str(seis_w.get("directory", "."))
        out_fmt = str(seis_w.get("format", "ascii")).lower()
    wave_w = (mode.get("writer", {}) or {}).get("wavefield", {}) or {}
    wf = {}
    if wave_w:
        if "time-interval-by-memory" in wave_w:
            raise ValueError("wavefield writer: time-interval-by-memory is not on this path")
        if bool(wave_w.get("for-adjoint-simulations", False)):
            raise ValueError("wavefield writer: stored boundary values for a reconstructed backward run "
                             "are not on this path (the adjoint recomputes from checkpoints)")
        fmt = str(wave_w.get("format", "ascii")).lower()
        if fmt not in ("ascii", "npy"):
            raise ValueError(f"wavefield writer: format {fmt!r} is not on this path (ASCII or NPY)")
        wf = dict(wavefield_directory=str(wave_w.get("directory", ".")), wavefield_format=fmt,
                  wavefield_interval=int(wave_w.get("time-interval", 0)),
                  wavefield_last_step=bool(wave_w.get("include-last-step", True)))
    types = [str(t).lower() for t in rc.get("seismogram-type", ["displacement"])]
    for t in types:
        if t not in EXT:
            raise ValueError(f"seismogram type {t!r} is not on this path")
    return ForwardConfig(dt=float(ts["dt"]), nstep=int(ts["nstep"]), elastic_wave="sh" if wave == "SH" else "psv",
                         database=_resolve(cfg["databases"]["mesh-database"], roots),
                         sources=(cfg["sources"] if isinstance(cfg["sources"], dict)
                                  else _resolve(cfg["sources"], roots)),
                         stations=(rc["stations"] if isinstance(rc["stations"], list)
                                   else _resolve(rc["stations"], roots)),
                         angle=float(rc.get("angle", 0.0)), seismogram_types=types,
                         nstep_between_samples=int(rc.get("nstep_between_samples", 1)),
                         output_directory=out_dir, output_format=out_fmt,
                         start_time=float(ts["t0"]) if "t0" in ts else None, **wf)


def read_stations(path):
    """2D STATIONS: (network, station) names and x, z coordinates; ``path``
    may also be the configuration's YAML list of stations (network, station,
    x, z), the reference's second form (src/io/receivers/dim2/read_receivers.cpp)."""
    if isinstance(path, list):
        if not path:
            raise ValueError("No receiver stations found in the YAML file")
        names = [(str(st["network"]), str(st["station"])) for st in path]
        return (names, np.asarray([float(st["x"]) for st in path], np.float64),
                np.asarray([float(st["z"]) for st in path], np.float64))
    names, xs, zs = [], [], []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) < 4 or p[0].startswith("#"):
                continue
            names.append((p[1], p[0]))
            xs.append(float(p[2]))
            zs.append(float(p[3]))
    return names, np.asarray(xs, np.float64), np.asarray(zs, np.float64)


def load_sources_node(path):
    """The sources node: a ``sources.yaml`` file, or the node given inline in
    the configuration (the reference tries the file first, then the node:
    src/io/sources/dim2/read_sources.cpp, dim3/read_sources.cpp)."""
    if isinstance(path, dict):
        return path
    import yaml
    with open(path) as f:
        return yaml.safe_load(f)


def read_sources(path):
    """Sources of a ``sources.yaml`` (or an inline sources node) as
    ``sfg.Source`` objects."""
    from .sfg import Source
    d = load_sources_node(path)
    out = []
    for s in d["sources"]:
        if "force" in s:
            fs, kind = s["force"], "force"
        elif "moment-tensor" in s:
            fs, kind = s["moment-tensor"], "moment_tensor"
        else:
            raise ValueError(f"source type {list(s)} is not on this path")
        tf, stf = time_function(fs)
        out.append(Source(x=float(fs["x"]), z=float(fs["z"]), f0=float(tf.get("f0", 0.0)),
                          factor=float(tf["factor"]), tshift=float(tf.get("tshift", 0.0)),
                          angle=float(fs.get("angle", 0.0)), stf=stf, kind=kind,
                          mxx=float(fs.get("Mxx", 0.0)), mzz=float(fs.get("Mzz", 0.0)),
                          mxz=float(fs.get("Mxz", 0.0)), hdur=float(tf.get("hdur", 0.0))))
    return out


def time_function(fs):
    """(parameters, kind) of a source's time function block
    (core/specfem/source/source.tpp:10-70): Ricker, Dirac, Gaussian (by f0
    or by hdur), dGaussian, Heaviside."""
    for key, kind in (("Ricker", "ricker"), ("Dirac", "dirac"), ("dGaussian", "dgaussian"),
                      ("Heaviside", "heaviside")):
        if key in fs:
            return fs[key], kind
    if "Gaussian" in fs:
        g = fs["Gaussian"]
        if "hdur" in g:
            return g, "gaussian_hdur"
        if "f0" in g:
            return g, "gaussian"
        raise ValueError("a Gaussian time function needs hdur or f0")
    raise ValueError("source time function not on this path (Ricker, Dirac, Gaussian, dGaussian, Heaviside)")


def channels(kind: str, elastic_wave: str):
    if kind in ("rotation", "intrinsic_rotation", "curl"):
        return ["BXY"]                       # Cosserat scalar traces
    if kind == "pressure":
        if elastic_wave == "sh":
            raise ValueError("pressure seismograms are not defined for SH waves")
        return ["PRE"]
    return ["BXY"] if elastic_wave == "sh" else ["BXX", "BXZ"]


def write_seismograms_ascii(directory: str, stations, seis, types, t0: float, dt: float, nsb: int,
                            elastic_wave: str = "psv"):
    """Write ``seis`` [nsig, ntypes, nrec, 2] as reference-format ASCII traces;
    returns the written paths."""
    os.makedirs(directory, exist_ok=True)
    paths = []
    nsig = seis.shape[0]
    t = t0 + np.arange(nsig, dtype=np.float64) * dt * nsb
    for r, (net, sta) in enumerate(stations):
        for k, kind in enumerate(types):
            for c, ch in enumerate(channels(kind, elastic_wave)):
                p = os.path.join(directory, f"{net}.{sta}.S2.{ch}.{EXT[kind]}")
                v = seis[:, k, r, c].astype(np.float64)
                with open(p, "w") as f:
                    f.writelines(f"{ti:e} {vi:e}\n" for ti, vi in zip(t, v))
                paths.append(p)
    return paths


# ---------------------------------------------------------------------------
# Output libraries of the reference (folders, groups and datasets).
#
# A "file" and each "group" in it are folders (an existing one is replaced);
# a dataset is, for the ASCII library, ``<name>.txt`` with one value per line
# (reals as %.10e with magnitudes below the type's smallest normal written as
# 0, integers as %d, booleans as 0 / 1) plus ``<name>.meta`` ("rank R" and
# "dims d0 d1 ..."), include/io/ASCII/impl/datasetbase.hpp and native_type.tpp;
# for the NPY library ``<name>.npy`` whose header declares Fortran order and
# the dataset's dims, include/io/NPY/impl/datasetbase.hpp.  Values are
# written in the memory order of the reference's view: LayoutLeft views
# (fields [nglob][ncomp], the element-to-point mapping) column-major, and the
# element-tiled views of kernels and coordinates ([nspec][ngllz][ngllx],
# include/domain_view.hpp:138-168, tiles of one element in a CPU build)
# element by element with iz fastest inside an element.

_DESCR = {np.dtype(np.float32): "<f4", np.dtype(np.float64): "<f8", np.dtype(np.int32): "<i4",
          np.dtype(np.bool_): "|b1"}


def _new_folder(path: str) -> str:
    if os.path.exists(path):
        shutil.rmtree(path)
    os.mkdir(path)
    return path


def _ascii_value_lines(flat: np.ndarray):
    if flat.dtype == np.bool_:
        return (("1" if v else "0") + "\n" for v in flat)
    if np.issubdtype(flat.dtype, np.integer):
        return (f"{int(v)}\n" for v in flat)
    tiny = np.finfo(flat.dtype).tiny
    vals = np.where(np.abs(flat) < tiny, 0.0, flat.astype(np.float64))
    return (f"{v:.10e}\n" for v in vals)


def write_dataset(folder: str, name: str, flat, dims, library: str = "ascii") -> str:
    """Write one dataset: ``flat`` holds the values in the view's memory order,
    ``dims`` its extents.  Returns the data file's path."""
    flat = np.ascontiguousarray(flat).ravel()
    dims = [int(d) for d in dims]
    if int(np.prod(dims)) != flat.size:
        raise ValueError(f"dataset {name}: {flat.size} values for dims {dims}")
    if library == "ascii":
        with open(os.path.join(folder, name + ".meta"), "w") as f:
            f.write(f"rank {len(dims)}\n")
            f.write("dims " + "".join(f"{d} " for d in dims) + "\n")
        path = os.path.join(folder, name + ".txt")
        with open(path, "w") as f:
            f.writelines(_ascii_value_lines(flat))
        return path
    if library == "npy":
        path = os.path.join(folder, name + ".npy")
        header = {"descr": _DESCR[flat.dtype], "fortran_order": True, "shape": tuple(dims)}
        with open(path, "wb") as f:
            np.lib.format.write_array_header_1_0(f, header)
            f.write(flat.tobytes())
        return path
    raise ValueError(f"unknown output library {library!r} (ascii or npy)")


def read_dataset(folder: str, name: str, dtype=np.float32):
    """Read a dataset written by ``write_dataset`` (or by the reference's
    ASCII / NPY libraries): (values in file order, dims)."""
    npy = os.path.join(folder, name + ".npy")
    if os.path.exists(npy):
        with open(npy, "rb") as f:
            version = np.lib.format.read_magic(f)
            read_header = (np.lib.format.read_array_header_1_0 if version == (1, 0)
                           else np.lib.format.read_array_header_2_0)
            shape, _, dt = read_header(f)
            flat = np.frombuffer(f.read(), dtype=dt)
        return flat, list(shape)
    with open(os.path.join(folder, name + ".meta")) as f:
        meta = dict(line.split(None, 1) for line in f if line.strip())
    dims = [int(v) for v in meta["dims"].split()]
    with open(os.path.join(folder, name + ".txt")) as f:
        flat = np.array([float(v) for v in f if v.strip()], dtype=np.float64)
    return flat.astype(dtype), dims


def element_order(a) -> np.ndarray:
    """[nspec, 25] (point q = iz*5 + ix) -> memory order of the reference's
    element-tiled [nspec][ngllz][ngllx] view in a CPU build (per element, iz
    fastest)."""
    a = np.asarray(a)
    return a.reshape(-1, 5, 5).transpose(0, 2, 1).ravel()


def from_element_order(flat) -> np.ndarray:
    """Inverse of ``element_order``: [nspec, 25]."""
    return np.asarray(flat).reshape(-1, 5, 5).transpose(0, 2, 1).reshape(-1, 25)


def geometry_of(source):
    """(x, z, |J| [nspec, 25], medium [nspec]) of a Simulation2D (from the
    library) or of a mesh with control nodes (meshgen.gll_geometry)."""
    if hasattr(source, "geometry"):
        return source.geometry()
    from .meshgen import gll_geometry
    x, z, jac = gll_geometry(source)
    return x, z, jac, np.asarray(source.mat_medium)[np.asarray(source.kmato)]


def _medium_elements(medium):
    """Database elements of each medium: {"elastic": idx, "acoustic": idx}."""
    medium = np.asarray(medium)
    return {"elastic": np.nonzero(medium == 1)[0], "acoustic": np.nonzero(medium == 0)[0]}


def isotropic_kernels(rho, kappa, mu, grad_rho, grad_kappa, grad_mu, jac):
    """Relative (logarithmic) Frechet kernel densities per element GLL point
    from the gradient of a misfit with respect to the point values of rho,
    kappa and mu ([nspec, 25] each, kappa the bulk modulus the medium
    stores): K_m = m (dL/dm) / (w_x w_z |J|), and the derived rho' = K_rho +
    K_kappa + K_mu, alpha = 2 (1 + 4 mu / (3 kappa)) K_kappa and beta = 2 (K_mu
    - 4 mu / (3 kappa) K_kappa) (Tromp et al. 2005, Eq. 20; the reference's
    include/medium/dim2/elastic/isotropic/frechet_derivative.hpp:164-180, whose
    prefactors use lambda + mu where this uses the stored bulk modulus).
    Returns a dict of [nspec, 25] arrays named as the reference's kernels."""
    from .meshgen import GLL_WEIGHTS
    w = np.outer(GLL_WEIGHTS, GLL_WEIGHTS).ravel()[None, :] * np.asarray(jac, np.float64)
    rho, kappa, mu = (np.asarray(v, np.float64) for v in (rho, kappa, mu))
    k_rho = rho * np.asarray(grad_rho, np.float64) / w
    k_kappa = kappa * np.asarray(grad_kappa, np.float64) / w
    k_mu = mu * np.asarray(grad_mu, np.float64) / w
    return {"rho": k_rho, "mu": k_mu, "kappa": k_kappa, "rhop": k_rho + k_kappa + k_mu,
            "alpha": 2.0 * (1.0 + 4.0 / 3.0 * mu / kappa) * k_kappa,
            "beta": 2.0 * (k_mu - 4.0 / 3.0 * mu / kappa * k_kappa)}


def write_kernels(output_folder: str, source, kernels, library: str = "ascii",
                  group: str = "elastic_psv_isotropic", dtype=np.float32) -> str:
    """Write per-element-point kernels ({name: [nspec, 25]}, e.g. from
    ``isotropic_kernels``) of the elements of ``group``'s medium as
    ``<output_folder>/Kernels/<group>/{X, Z, <name>...}`` with dims [n][5][5]
    (include/io/impl/medium_writer.tpp); ``source`` gives the geometry
    (``geometry_of``).  Returns the Kernels folder."""
    x, z, _, medium = geometry_of(source)
    elems = _medium_elements(medium)["acoustic" if group.startswith("acoustic") else "elastic"]
    os.makedirs(output_folder, exist_ok=True)
    root = _new_folder(os.path.join(output_folder, "Kernels"))
    g = _new_folder(os.path.join(root, group))
    n = len(elems)
    write_dataset(g, "X", element_order(x[elems]).astype(dtype), (n, 5, 5), library)
    write_dataset(g, "Z", element_order(z[elems]).astype(dtype), (n, 5, 5), library)
    for name, v in kernels.items():
        v = np.asarray(v).reshape(-1, 25)
        write_dataset(g, name, element_order(v[elems]).astype(dtype), (n, 5, 5), library)
    return root


class WavefieldWriter:
    """Forward-wavefield snapshots in the layout of the reference's wavefield
    writer (include/io/wavefield/writer.tpp):
    ``<output_folder>/ForwardWavefield/Coordinates/<medium>/{X, Z, mapping}``
    (X, Z per point of the medium, mapping [n][5][5] element point -> point),
    ``Step<6-digit step>/<medium>/{Displacement, Velocity, Acceleration}``
    ([nglob][ncomp], LayoutLeft) or ``{Potential, PotentialDot,
    PotentialDotDot}`` for the acoustic medium, and
    ``BoundaryValues/save_boundary_values`` (false: the adjoint here
    recomputes from checkpoints instead of replaying stored boundary values).
    The point numbering is the handle's; ``mapping`` ties it to the elements.
    The geometry comes from ``mesh`` when given, else from the handle."""

    def __init__(self, output_folder: str, sim, mesh=None, library: str = "ascii"):
        self.sim, self.library = sim, library
        self.geometry = geometry_of(sim if mesh is None else mesh)
        self.root = os.path.join(output_folder, "ForwardWavefield")
        wave = "elastic_sh" if getattr(sim, "ncomp", 2) == 1 else "elastic_psv"
        self.names = {"elastic": wave, "acoustic": "acoustic"}

    def initialize(self):
        os.makedirs(os.path.dirname(self.root), exist_ok=True)
        _new_folder(self.root)
        coords = _new_folder(os.path.join(self.root, "Coordinates"))
        ib, g2e, g2a = self.sim.numbering()
        x, z, _, med = self.geometry
        for medium, elems in _medium_elements(med).items():
            if len(elems) == 0:
                continue
            g2m = g2e if medium == "elastic" else g2a
            mapping = g2m[ib[elems]]                                   # [n, 25]
            npts = int(mapping.max()) + 1
            px = np.zeros(npts, np.float32)
            pz = np.zeros(npts, np.float32)
            px[mapping.ravel()] = x[elems].ravel()
            pz[mapping.ravel()] = z[elems].ravel()
            g = _new_folder(os.path.join(coords, self.names[medium]))
            write_dataset(g, "X", px, (npts,), self.library)
            write_dataset(g, "Z", pz, (npts,), self.library)
            m3 = mapping.reshape(-1, 5, 5)                               # [iel][iz][ix]
            write_dataset(g, "mapping", m3.transpose(2, 1, 0).ravel().astype(np.int32),
                          m3.shape, self.library)

    def write(self, istep: int):
        base = _new_folder(os.path.join(self.root, f"Step{istep:06d}"))
        for medium, elems in _medium_elements(self.geometry[3]).items():
            if len(elems) == 0:
                continue
            g = _new_folder(os.path.join(base, self.names[medium]))
            names = (("Potential", "PotentialDot", "PotentialDotDot") if medium == "acoustic"
                     else ("Displacement", "Velocity", "Acceleration"))
            for which, name in zip(("displacement", "velocity", "acceleration"), names):
                f = np.asarray(self.sim.field(medium, which), np.float32)
                f2 = f.reshape(f.shape[0], -1)                           # [nglob][ncomp]
                write_dataset(g, name, f2.T.ravel(), f2.shape, self.library)

    def finalize(self):
        b = _new_folder(os.path.join(self.root, "BoundaryValues"))
        write_dataset(b, "save_boundary_values", np.array([False]), (1,), self.library)
