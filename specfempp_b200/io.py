"""Reference-format inputs and outputs of the 2D forward run.

* ``read_config``: the subset of a SPECFEM++ ``specfem_config.yaml`` that a
  forward Newmark run needs (src/parameter_parser/setup.cpp and the
  ``parameters`` keys of the reference's example configurations);
* ``read_stations``: a 2D STATIONS file (station, network, x, z, ...);
* ``read_sources``: a ``sources.yaml`` with force and moment-tensor sources,
  Ricker or Dirac time functions (src/io/sources/dim2/read_sources.cpp);
* ``write_seismograms_ascii``: one two-column ``time value`` file per station,
  component and seismogram type, named ``NET.STA.S2.<channel>.<ext>`` like the
  reference's writer (src/io/seismogram/writer.cpp:8-141).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

EXT = {"displacement": "semd", "velocity": "semv", "acceleration": "sema", "pressure": "semp"}


@dataclass
class ForwardConfig:
    dt: float
    nstep: int
    elastic_wave: str                 # "psv" or "sh"
    database: str                     # path of database.bin
    sources: str                      # path of sources.yaml
    stations: str                     # path of STATIONS
    angle: float = 0.0
    seismogram_types: list = field(default_factory=lambda: ["displacement"])
    nstep_between_samples: int = 1
    output_directory: str = "."
    output_format: str = "ascii"


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
    types = [str(t).lower() for t in rc.get("seismogram-type", ["displacement"])]
    for t in types:
        if t not in EXT:
            raise ValueError(f"seismogram type {t!r} is not on this path")
    return ForwardConfig(dt=float(ts["dt"]), nstep=int(ts["nstep"]), elastic_wave="sh" if wave == "SH" else "psv",
                         database=_resolve(cfg["databases"]["mesh-database"], roots),
                         sources=_resolve(cfg["sources"], roots), stations=_resolve(rc["stations"], roots),
                         angle=float(rc.get("angle", 0.0)), seismogram_types=types,
                         nstep_between_samples=int(rc.get("nstep_between_samples", 1)),
                         output_directory=out_dir, output_format=out_fmt)


def read_stations(path: str):
    """2D STATIONS: (network, station) names and x, z coordinates."""
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


def read_sources(path: str):
    """Sources of a ``sources.yaml`` as ``sfg.Source`` objects."""
    import yaml
    from .sfg import Source
    with open(path) as f:
        d = yaml.safe_load(f)
    out = []
    for s in d["sources"]:
        if "force" in s:
            fs, kind = s["force"], "force"
        elif "moment-tensor" in s:
            fs, kind = s["moment-tensor"], "moment_tensor"
        else:
            raise ValueError(f"source type {list(s)} is not on this path")
        if "Ricker" in fs:
            tf, stf = fs["Ricker"], "ricker"
        elif "Dirac" in fs:
            tf, stf = fs["Dirac"], "dirac"
        else:
            raise ValueError("only Ricker and Dirac source time functions are on this path")
        out.append(Source(x=float(fs["x"]), z=float(fs["z"]), f0=float(tf.get("f0", 0.0)),
                          factor=float(tf["factor"]), tshift=float(tf.get("tshift", 0.0)),
                          angle=float(fs.get("angle", 0.0)), stf=stf, kind=kind,
                          mxx=float(fs.get("Mxx", 0.0)), mzz=float(fs.get("Mzz", 0.0)),
                          mxz=float(fs.get("Mxz", 0.0))))
    return out


def channels(kind: str, elastic_wave: str):
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
