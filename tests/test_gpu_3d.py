"""3D elastic CUDA path against the 3D oracle and the reference's dim3 golden
traces.

Tolerances (fixed): displacement and velocity relative L2 <= 1e-5 against
the oracle FP32, acceleration <= 1e-4 (FP32 noise floor, as in
test_gpu_parity); golden traces sum|d|/sum|ref| < 1e-3 per station.
"""
import numpy as np
import pytest

from conftest import rel_l2
from test_oracle import golden3d_case

pytestmark = pytest.mark.gpu

TYPES = ("displacement", "velocity", "acceleration")


def product3d(case, epb=0, types=TYPES, variant=0):
    from specfempp_b200 import sfg3d
    sim = sfg3d.Simulation3D(case.mesh, dt=case.dt, nstep=case.nstep, elements_per_block=epb,
                             kernel_variant=variant)
    sim.set_sources(case.sources)
    sim.set_receivers(case.rec_xyz, types=types)
    sim.initialize()
    sim.run(case.nstep)
    return sim, sim.seismograms()


def tol(kind, f32=None, f64=None):
    return 1e-5 if kind in ("displacement", "velocity") else 1e-4


def test_3d_golden_fixture(sfg_lib, oracle_lib):
    from oracle import runner3d
    case, z = golden3d_case()
    case.seis_types = list(TYPES)
    ref = runner3d.run(case, "f32", nthreads=8)["seis"]
    ref64 = runner3d.run(case, "f64", nthreads=8)["seis"]
    sim, seis = product3d(case)
    assert sim.check_finite()
    for t, (kind, key) in enumerate(zip(TYPES, ("traces_semd", "traces_semv", "traces_sema"))):
        assert rel_l2(seis[:, t], ref[:, t]) <= tol(kind, ref[:, t], ref64[:, t]), (kind, rel_l2(seis[:, t], ref[:, t]))
        c = np.transpose(seis[:, t], (1, 2, 0))
        tr = z[key]
        err = np.abs(c - tr).sum(axis=(1, 2)) / np.abs(tr).sum(axis=(1, 2))
        assert err.max() < 1e-3, (kind, err.max())


def small_absorbing_case(nstep=300):
    from oracle import runner3d
    from specfempp_b200 import meshgen
    w = meshgen.elastic3d_layered_grf(nex=10, ney=8, nez=6, nstep=nstep, nrec=12, seed=3)
    s = w.sources[0]
    src = [runner3d.Source3D(s.x, s.y, s.z, f0=4.0, factor=1e13, kind=s.kind, comp=s.comp),
           runner3d.Source3D(0.3 * 5000, 0.6 * 4000, -1500.0, f0=3.0, factor=1e12, kind="force",
                             comp=(0.3, -0.5, 1.0, 0, 0, 0), tshift=0.05)]
    return runner3d.Case3D(w.mesh, src, w.rec_xyz, 2e-3, nstep, list(TYPES))


def test_3d_absorbing_moment_tensor_vs_oracle(sfg_lib, oracle_lib):
    """Layered GRF model, Stacey on five faces, free top, a moment tensor and
    a force source with a time shift: all three seismogram types and the final
    displacement field against the oracle."""
    from oracle import runner3d
    case = small_absorbing_case()
    r = runner3d.run(case, "f32", nthreads=8, want_final=True)
    r64 = runner3d.run(case, "f64", nthreads=8)
    sim, seis = product3d(case, epb=2)
    assert np.abs(r["seis"]).max() > 0
    for t, kind in enumerate(TYPES):
        assert rel_l2(seis[:, t], r["seis"][:, t]) <= tol(kind, r["seis"][:, t], r64["seis"][:, t]), kind
    assert rel_l2(sim.field("displacement"), r["final"]) <= 1e-5


def test_3d_launch_shapes_agree_and_deterministic(sfg_lib):
    """Point form (1, 2, 4 elements per block) and column form (6, 8): the
    same bits, seismograms and final field, with sources and absorbing
    faces."""
    case = small_absorbing_case(nstep=120)
    s1, a = product3d(case, epb=1)
    _, b = product3d(case, epb=4)
    for e in (6, 8):
        sc, d = product3d(case, epb=e)
        assert sc.info().kernel_variant == 2
        assert np.array_equal(a, d), e
        assert np.array_equal(s1.field("displacement"), sc.field("displacement")), e
    sim, c = product3d(case, epb=2)
    assert np.array_equal(a, b) and np.array_equal(a, c)
    sim.reset()
    sim.run(case.nstep)
    assert np.array_equal(sim.seismograms(), c)


def test_3d_absorbing_energy_decays(sfg_lib):
    """Absorbing faces take the (resolved, 1 Hz) wavefield out of the model:
    late-time receiver energy falls below 1e-3 of its peak and far below the
    same run with free faces everywhere."""
    from specfempp_b200 import meshgen, sfg3d
    from oracle import runner3d
    late = {}
    for absorb in (0, 1):
        m = meshgen.homogeneous_hex_mesh(8, 8, 8, (0, 4000, 0, 4000, -4000, 0), 2500.0, 3000.0, 1732.0,
                                         absorbing=(absorb,) * 6)
        src = [runner3d.Source3D(2000.0, 2000.0, -2000.0, f0=1.0, factor=1e12, comp=(0, 0, 1.0, 0, 0, 0))]
        sim = sfg3d.Simulation3D(m, dt=4e-3, nstep=1500)
        sim.set_sources(src)
        sim.set_receivers(np.array([[2000.0, 2000.0, -1000.0], [500.0, 500.0, -500.0]]), types=("velocity",))
        sim.initialize()
        sim.run(1500)
        e = (sim.seismograms()[:, 0].astype(np.float64) ** 2).sum(axis=(1, 2))
        late[absorb] = (e[1200:].max(), e.max())
    assert late[1][0] < 1e-3 * late[1][1]
    assert late[1][0] < 1e-2 * late[0][0]


def test_specfem3d_config_driver(sfg_lib, oracle_lib, tmp_path):
    """The 3D configuration driver on the dim3 fixture's own run directory
    (its database.bin, STATIONS and force.yaml): the written
    ``NET.STA.S3.BX?.sem?`` traces against the golden SPECFEM3D traces
    (sum|d|/sum|ref| < 1e-3 per station) and against the oracle FP32 on the
    mesh read from the database (relative L2 as above)."""
    import os
    from conftest import GOLDEN
    from fixture_dir import write_fixture_dir3d
    from oracle import runner3d
    from specfempp_b200 import database3d, specfem3d
    cfg, z = write_fixture_dir3d(os.path.join(GOLDEN, "HomogeneousHalfspaceSmallNoABCForceSource.npz"),
                                 str(tmp_path))
    out = specfem3d.run_config(cfg, root=str(tmp_path))
    assert out["lattice"] == [8, 6, 6] and out["files"] == len(z["stations"]) * 3 * 3
    mesh = database3d.lattice_mesh(database3d.read_database3d(str(tmp_path / "database.bin")))
    (s,) = specfem3d.read_sources3d(str(tmp_path / "force.yaml"))
    case = runner3d.Case3D(mesh, [runner3d.Source3D(s.x, s.y, s.z, f0=s.f0, factor=s.factor, kind=s.kind,
                                                    comp=s.comp, tshift=s.tshift)],
                           z["rec_xyz"], float(z["dt"]), int(z["nstep"]), list(TYPES))
    ref = runner3d.run(case, "f32", nthreads=8)["seis"]           # [nstep, ntypes, nrec, 3]
    for t, (kind, ext) in enumerate(zip(TYPES, ("semd", "semv", "sema"))):
        got = np.zeros((len(z["stations"]), 3, int(z["nstep"])))
        for r, st in enumerate(z["stations"]):
            for c, ch in enumerate(("BXX", "BXY", "BXZ")):
                tt, v = np.loadtxt(os.path.join(out["output_directory"], f"{st}.S3.{ch}.{ext}")).T
                assert abs(tt[0] - float(z["trace_t0"])) < 1e-6
                got[r, c] = v
        tr = z[f"traces_{ext}"]
        err = np.abs(got - tr).sum(axis=(1, 2)) / np.abs(tr).sum(axis=(1, 2))
        assert err.max() < 1e-3, (kind, err.max())
        # the files hold 7 significant digits (%e), well inside the bar
        assert rel_l2(np.transpose(got, (2, 0, 1)), ref[:, t]) <= tol(kind), kind
