"""Command-line forward run from a reference configuration (GPU path).

    python -m specfempp_b200.specfem2d -p specfem_config.yaml [--root DIR]

Reads the reference's ``specfem_config.yaml`` (forward, Newmark), its
``database.bin`` (xmeshfem2D output), ``sources.yaml`` and ``STATIONS``, runs
the time loop on the GPU through libsfg, and writes the seismograms as the
reference's ASCII traces (``NET.STA.S2.BXX.semd`` ...), and, when the
configuration has a wavefield writer, the forward wavefield every
``time-interval`` steps and at the last step in the reference's
``ForwardWavefield`` layout (ASCII or NPY).  This mirrors the
reference's ``specfem2d -p <config>`` program (src/specfem2d.cpp,
core/specfem/program) for the forward 2D path.
"""
from __future__ import annotations

import argparse
import json
import os
import time

from . import io
from .sfg import Simulation2D


def run_config(config: str, root: str | None = None, output_directory: str | None = None) -> dict:
    cfg = io.read_config(config, root)
    sources = io.read_sources(cfg.sources)
    stations, rx, rz = io.read_stations(cfg.stations)
    t = time.perf_counter()
    sim = Simulation2D(database=cfg.database, dt=cfg.dt, nstep=cfg.nstep,
                       nstep_between_samples=cfg.nstep_between_samples, elastic_wave=cfg.elastic_wave,
                       start_time=cfg.start_time)
    sim.set_sources(sources)
    sim.set_receivers(rx, rz, angle=cfg.angle, types=tuple(cfg.seismogram_types))
    sim.initialize()
    setup_s = time.perf_counter() - t
    writer = None
    if cfg.wavefield_directory is not None:
        wdir = cfg.wavefield_directory
        if not os.path.isabs(wdir):
            wdir = os.path.join(root or os.getcwd(), wdir)
        if not os.path.isdir(wdir):
            raise FileNotFoundError(f"Output folder : {wdir} does not exist.")
        writer = io.WavefieldWriter(wdir, sim, library=cfg.wavefield_format)
        writer.initialize()
    t = time.perf_counter()
    written = []
    if writer is not None and cfg.wavefield_interval > 0:
        # snapshots after every time_interval steps (periodic_task.hpp:59-69)
        done = 0
        while done < cfg.nstep:
            n = min(cfg.wavefield_interval - done % cfg.wavefield_interval, cfg.nstep - done)
            sim.run(n)
            done += n
            if done % cfg.wavefield_interval == 0:
                writer.write(done)
                written.append(done)
    else:
        sim.run(cfg.nstep)
    if writer is not None:
        if cfg.wavefield_last_step and cfg.nstep not in written:
            writer.write(cfg.nstep)
            written.append(cfg.nstep)
        writer.finalize()
    seis = sim.seismograms()[0]
    run_s = time.perf_counter() - t
    inf = sim.info()
    out_dir = output_directory or cfg.output_directory
    if not os.path.isabs(out_dir):
        out_dir = os.path.join(root or os.getcwd(), out_dir)
    paths = io.write_seismograms_ascii(out_dir, stations, seis, cfg.seismogram_types, inf.t0, cfg.dt,
                                       cfg.nstep_between_samples, cfg.elastic_wave)
    sim.close()
    return {"nspec": inf.nspec, "nglob": inf.nglob, "nstep": cfg.nstep, "setup_s": setup_s, "run_s": run_s,
            "files": len(paths), "output_directory": out_dir, "wavefield_steps": written}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-p", "--parameters", required=True, help="specfem_config.yaml")
    ap.add_argument("--root", default=None, help="directory the configuration's relative paths start from")
    ap.add_argument("-o", "--output", default=None, help="seismogram directory (overrides the configuration)")
    a = ap.parse_args(argv)
    print(json.dumps(run_config(a.parameters, a.root, a.output)))


if __name__ == "__main__":
    main()
