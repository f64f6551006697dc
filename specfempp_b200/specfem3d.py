"""Command-line 3D forward run from a reference configuration (GPU path).

    python -m specfempp_b200.specfem3d -p specfem_config.yaml [--root DIR] [--absorbing]

Reads the reference's 3D ``specfem_config.yaml`` (forward, Newmark), its mesh
``database.bin`` (the 3D mesher's output, ``database3d``), the sources YAML
(force and moment-tensor sources with Ricker time functions) and the 3D
``STATIONS`` file (station, network, y, x, elevation, z), runs the time loop
on the GPU through the 3D library, and writes the seismograms as the
reference's ASCII traces ``NET.STA.S3.<band>X{X,Y,Z}.<ext>``.  This mirrors
the reference's 3D program (core/specfem/program/program.cpp:269-423,
src/specfem3d.cpp): its source reader (src/io/sources/dim3/read_sources.cpp,
start time t0 = min over sources of -1.2/f0 + tshift), its receiver reader
(src/io/receivers/dim3/read_receivers.cpp) and its seismogram writer
(src/io/seismogram/writer.cpp:143-186 with the SEED band code of
src/io/seismogram/impl/channel_generator.cpp).  The reference's 3D path has
no absorbing boundary; ``--absorbing`` adds the library's Stacey condition on
the sides the database lists, the top excepted.
"""
from __future__ import annotations

import argparse
import json
import os
import time
from dataclasses import dataclass

import numpy as np

from . import database3d, io
from .sfg3d import Simulation3D

TYPES3D = ("displacement", "velocity", "acceleration")


@dataclass
class Source3DSpec:
    x: float
    y: float
    z: float
    f0: float
    factor: float
    tshift: float
    kind: str           # "force" or "moment_tensor"
    comp: tuple         # (fx, fy, fz, 0, 0, 0) or (Mxx, Myy, Mzz, Mxy, Mxz, Myz)


def read_stations3d(path):
    """3D STATIONS lines ``station network y x elevation z`` (the y and x
    columns are latitude-like and longitude-like): (network, station) names
    and [nrec, 3] (x, y, z).  ``path`` may also be the configuration's YAML
    list of stations (network, station, x, y, z)."""
    if isinstance(path, list):
        if not path:
            raise ValueError("No receiver stations found in the YAML file")
        return ([(str(st["network"]), str(st["station"])) for st in path],
                np.asarray([[float(st["x"]), float(st["y"]), float(st["z"])] for st in path], np.float64))
    names, xyz = [], []
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p or p[0].startswith("#"):
                continue
            if len(p) != 6:
                raise ValueError(f"STATIONS line {line.strip()!r}: 6 columns expected (station network y x elev z)")
            names.append((p[1], p[0]))
            xyz.append((float(p[3]), float(p[2]), float(p[5])))
    return names, np.asarray(xyz, np.float64).reshape(-1, 3)


def read_sources3d(path):
    """Force (x, y, z, fx, fy, fz) and moment-tensor (x, y, z, Mxx, Myy, Mzz,
    Mxy, Mxz, Myz) sources with a Ricker time function, from a sources file
    or the sources node given inline in the configuration."""
    d = io.load_sources_node(path)
    out = []
    for s in d["sources"]:
        if "force" in s:
            fs, kind = s["force"], "force"
            comp = (float(fs["fx"]), float(fs["fy"]), float(fs["fz"]), 0.0, 0.0, 0.0)
        elif "moment-tensor" in s:
            fs, kind = s["moment-tensor"], "moment_tensor"
            comp = tuple(float(fs[k]) for k in ("Mxx", "Myy", "Mzz", "Mxy", "Mxz", "Myz"))
        else:
            raise ValueError(f"source type {list(s)} is not on the 3D path (force, moment-tensor)")
        if "Ricker" not in fs:
            raise ValueError("the 3D path takes Ricker source time functions")
        rk = fs["Ricker"]
        out.append(Source3DSpec(float(fs["x"]), float(fs["y"]), float(fs["z"]), float(rk["f0"]),
                                float(rk["factor"]), float(rk.get("tshift", 0.0)), kind, comp))
    n = int(d.get("number-of-sources", len(out)))
    if n != len(out):
        raise ValueError(f"Found only {len(out)} number of sources. Found total number of sources in are {n}")
    if not out:
        raise ValueError("No sources found in the sources file")
    return out


def subsample(seis, nsb: int):
    """The samples of steps 0, nsb, 2 nsb, ... of a run recorded every step
    (the reference records at istep % nstep_between_samples == 0)."""
    return seis[::max(1, int(nsb))]


def band_code(dt: float) -> str:
    """SEED band code of the sampling step (channel_generator.cpp)."""
    if dt >= 1.0:
        return "L"
    if dt >= 0.1:
        return "M"
    if dt > 0.0125:
        return "B"
    if dt > 0.004:
        return "H"
    if dt > 0.001:
        return "C"
    return "F"


def write_seismograms3d(directory: str, stations, seis, types, t0: float, dt: float, nsb: int):
    """``seis`` [nsig, ntypes, nrec, 3] as ``NET.STA.S3.<band>X<c>.<ext>``
    two-column ``time value`` files (%e, like std::scientific); returns the paths."""
    os.makedirs(directory, exist_ok=True)
    band = band_code(dt)
    t = t0 + np.arange(seis.shape[0], dtype=np.float64) * dt * nsb
    paths = []
    for r, (net, sta) in enumerate(stations):
        for k, kind in enumerate(types):
            for c, letter in enumerate("XYZ"):
                p = os.path.join(directory, f"{net}.{sta}.S3.{band}X{letter}.{io.EXT[kind]}")
                with open(p, "w") as f:
                    f.writelines(f"{ti:e} {vi:e}\n" for ti, vi in zip(t, seis[:, k, r, c].astype(np.float64)))
                paths.append(p)
    return paths


def run_config(config: str, root: str | None = None, output_directory: str | None = None,
               absorbing: bool = False, elements_per_block: int = 0) -> dict:
    cfg = io.read_config(config, root)
    if cfg.wavefield_directory is not None:
        raise ValueError("wavefield writers are not on the 3D path")
    if cfg.start_time is not None:
        raise ValueError("a user start time (time-scheme t0) is not on the 3D path")
    for t in cfg.seismogram_types:
        if t not in TYPES3D:
            raise ValueError(f"seismogram type {t!r} is not on the 3D path {TYPES3D}")
    if cfg.nstep_between_samples < 1:
        raise ValueError("nstep_between_samples must be at least 1")
    t = time.perf_counter()
    db = database3d.read_database3d(cfg.database)
    mesh = database3d.lattice_mesh(db, absorbing=absorbing)
    sources = read_sources3d(cfg.sources)
    stations, xyz = read_stations3d(cfg.stations)
    sim = Simulation3D(mesh, dt=cfg.dt, nstep=cfg.nstep, elements_per_block=elements_per_block)
    try:
        sim.set_sources(sources)
        sim.set_receivers(xyz, types=tuple(cfg.seismogram_types))
        sim.initialize()
        setup_s = time.perf_counter() - t
        t = time.perf_counter()
        sim.run(cfg.nstep)
        seis = sim.seismograms()
        run_s = time.perf_counter() - t
        inf = sim.info()
        if not sim.check_finite():
            raise FloatingPointError("the wavefield is not finite (unstable time step?)")
    finally:
        sim.close()
    out_dir = output_directory or cfg.output_directory
    if not os.path.isabs(out_dir):
        out_dir = os.path.join(root or os.getcwd(), out_dir)
    paths = write_seismograms3d(out_dir, stations, subsample(seis, cfg.nstep_between_samples),
                                cfg.seismogram_types, inf.t0, cfg.dt, cfg.nstep_between_samples)
    return {"nspec": inf.nspec, "nglob": inf.nglob, "lattice": [mesh.nex, mesh.ney, mesh.nez],
            "nstep": cfg.nstep, "setup_s": setup_s, "run_s": run_s, "files": len(paths),
            "output_directory": out_dir, "absorbing": list(mesh.absorbing)}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-p", "--parameters", required=True, help="specfem_config.yaml")
    ap.add_argument("--root", default=None, help="folder the configuration's relative paths start from")
    ap.add_argument("--output", default=None, help="seismogram folder (default: the configuration's)")
    ap.add_argument("--absorbing", action="store_true",
                    help="Stacey condition on the database's listed sides except the top")
    a = ap.parse_args(argv)
    print(json.dumps(run_config(a.parameters, a.root, a.output, a.absorbing)))


if __name__ == "__main__":
    main()
