"""The step-wise interface (the reference's kernel facade) and the compiled
C++ caller that reproduces time_marching<forward>::run over it.

* CPU: specfempp_b200/host/specfem2d_facade.cpp (with specfem_facade.hpp)
  compiles with g++ against include/sfg.h and links libsfg.so;
* GPU: the C++ time loop (predictor of both media, update_wavefields and
  corrector of the acoustic then the elastic medium, seismograms, and the
  reference's degree-of-freedom / element checks every step) gives
  sfg_run's seismograms bit for bit, on a coupled and an elastic model read
  from database.bin; the same calls through ctypes also leave sfg_run's
  end-of-step fields.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

STF_CODE = {"ricker": 0, "dirac": 1, "gaussian": 2, "gaussian_hdur": 3, "dgaussian": 4, "heaviside": 5}
TYPE_CODE = {"displacement": 0, "velocity": 1, "acceleration": 2, "pressure": 3}


def build_facade(tmp_path):
    from specfempp_b200 import build
    lib = build.build()
    exe = os.path.join(str(tmp_path), "specfem2d_facade")
    src = os.path.join(ROOT, "specfempp_b200", "host", "specfem2d_facade.cpp")
    libdir = os.path.dirname(lib)
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-o", exe, src, "-L" + libdir,
                    "-lsfg", "-Wl,-rpath," + libdir], check=True)
    return exe


def test_facade_compiles_against_the_header(tmp_path, sfg_lib):
    exe = build_facade(tmp_path)
    assert os.path.exists(exe)
    for name in ("sfg_predictor", "sfg_update_wavefields", "sfg_corrector", "sfg_compute_seismograms"):
        assert hasattr(sfg_lib, name)


def write_setup(path, w, nstep, types, nsb=1):
    with open(path, "w") as f:
        f.write(f"{w.dt!r} {nstep} {nsb} 0\n{len(w.sources)}\n")
        for s in w.sources:
            f.write(f"{s.x!r} {s.z!r} {s.f0!r} {s.factor!r} {getattr(s, 'tshift', 0.0)!r} "
                    f"{getattr(s, 'angle', 0.0)!r} {STF_CODE[getattr(s, 'stf', 'ricker')]}\n")
        f.write(f"{len(w.rec_x)} {len(types)} " + " ".join(str(TYPE_CODE[t]) for t in types) + "\n")
        for x, z in zip(w.rec_x, w.rec_z):
            f.write(f"{float(x)!r} {float(z)!r}\n")


def models():
    from specfempp_b200 import meshgen
    return {"coupled_80x40": meshgen.coupled_400x200(nstep=300, nx=80, nz=40),
            "elastic_80x60": meshgen.elastic_psv_80x60(nstep=300)}


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["coupled_80x40", "elastic_80x60"])
def test_cpp_time_loop_equals_sfg_run(tmp_path, sfg_lib, name):
    from specfempp_b200 import meshgen, sfg
    w = models()[name]
    nstep, types = 300, ("displacement", "velocity", "acceleration", "pressure")
    db = os.path.join(str(tmp_path), "database.bin")
    meshgen.write_database(w.mesh, db)
    setup = os.path.join(str(tmp_path), "setup.txt")
    write_setup(setup, w, nstep, types)
    out = os.path.join(str(tmp_path), "seis.bin")
    exe = build_facade(tmp_path)
    res = subprocess.run([exe, db, setup, out], capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    assert "elements" in res.stdout
    sim = sfg.Simulation2D(database=db, dt=w.dt, nstep=nstep)
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_x, w.rec_z, types=types)
    sim.initialize()
    sim.run(nstep)
    ref = sim.seismograms()[0]
    got = np.fromfile(out, np.float32).reshape(ref.shape)
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), float(np.abs(got - ref).max() / np.abs(ref).max())


@pytest.mark.gpu
def test_stepwise_calls_leave_sfg_run_fields(sfg_lib):
    """The step-wise calls in the reference's order, through ctypes, leave the
    fields sfg_run leaves (bit for bit) and return the reference's counts."""
    from specfempp_b200 import sfg
    w = models()["coupled_80x40"]
    nstep = 120
    sims = []
    for _ in range(2):
        s = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=nstep)
        s.set_sources(w.sources)
        s.set_receivers(w.rec_x, w.rec_z, types=("displacement", "velocity"))
        s.initialize()
        sims.append(s)
    a, b = sims
    a.run(nstep)
    inf = b.info()
    h = b.h
    AC, EL = 0, 1
    for istep in range(nstep):
        dofs = sfg_lib.sfg_predictor(h, AC) + sfg_lib.sfg_predictor(h, EL)
        elems = sfg_lib.sfg_update_wavefields(h, AC, istep)
        dofs += sfg_lib.sfg_corrector(h, AC)
        elems += sfg_lib.sfg_update_wavefields(h, EL, istep)
        dofs += sfg_lib.sfg_corrector(h, EL)
        assert sfg_lib.sfg_compute_seismograms(h, istep) == 0
        assert dofs == 2 * (inf.nglob_elastic * 2 + inf.nglob_acoustic)
        assert elems == inf.nspec
    b.synchronize()
    assert np.array_equal(a.seismograms(), b.seismograms())
    for med in ("elastic", "acoustic"):
        for f in ("displacement", "velocity", "acceleration"):
            assert np.array_equal(a.field(med, f), b.field(med, f)), (med, f)
    # out-of-range sample and bad medium are refused
    assert sfg_lib.sfg_compute_seismograms(h, nstep + 5) == -1
    assert sfg_lib.sfg_update_wavefields(h, 7, 0) == -1
