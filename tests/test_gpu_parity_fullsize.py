"""Full-size parity of the CUDA path with the CPU oracle on the benchmark
configurations, and the FP32 error of both against the FP64 oracle.

The oracle runs multithreaded with colour-ordered assembly (deterministic at
any thread count), in two FP32 evaluation orders of the same algorithm: the
device order (the 5-term contractions as fused multiply-adds, as the CUDA
kernels compute them; the checker) and the reference order (products and
sums rounded separately, as the reference's source is written), plus FP64.
Per configuration and output the test measures and records:

* CUDA FP32 vs oracle FP32 (device order, and reference order for
  configurations 1 and 2): displacement seismograms and elastic final fields
  <= 1e-5 (the parity bar of this path); velocity, elastic acceleration and the
  acoustic potential <= 1e-4; acceleration and pressure of the coupled model
  (acoustic-medium time derivatives) <= 5e-3.  The looser bounds are the
  measured FP32 noise floor: over thousands of steps each FP32 evaluation is
  4-5e-5 from FP64 in velocity and acceleration, two FP32 runs of different
  rounding differ by about 1.4 times that (up to 6e-5), and acoustic
  accelerations carry FP32 errors up to 1.4e-3 (see test_gpu_parity);
* CUDA FP32 vs FP64 <= 1.25 x (oracle FP32 vs FP64) + 1e-6: the CUDA build is
  as accurate as a CPU FP32 build of the reference.

With SFG_PARITY_RECORD=<path> every row is appended to that file as a JSON
line (the table in the design notes comes from it).

Configurations (seeded synthetic inputs of the benchmark shapes):
1. elastic P-SV 80x60, 1600 steps, 5 receivers (d, v, a) + final field;
2. coupled acoustic-elastic 400x200, 4000 steps, 200 receivers (d, v, a, p)
   + final fields of both media;
3. batched elastic 1000x500 GRF model, 32 shots in one run, 300 steps: the
   final fields of shots 0, 15 and 31 and the traces of shot 0 against
   single-shot oracle runs (FP64 for shot 0 only);
5. 3D elastic 128x128x64 hexahedra (67.6 M points), layered + GRF model,
   moment tensor: the final displacement field after 60 steps (10 Hz wavelet,
   so that the source has peaked inside the window).
"""
import json
import os
from dataclasses import replace

import numpy as np
import pytest

from conftest import oracle_f32, rel_l2, workload_case

pytestmark = pytest.mark.gpu

NT = max(1, os.cpu_count() or 1)
TOL_DV = 1e-5      # displacement seismograms, elastic final fields
TOL_AP = 1e-4      # velocity, elastic acceleration, acoustic potential (FP32 noise floor)
TOL_NOISY = 5e-3   # acceleration and pressure with receivers in an acoustic medium


def bound(quantity, coupled=False):
    base = quantity.split(":")[0]
    if base == "displacement" or (base == "field" and "acoustic" not in quantity):
        return TOL_DV
    if coupled and base in ("acceleration", "pressure"):
        return TOL_NOISY
    return TOL_AP


def record(row):
    print(json.dumps(row))
    path = os.environ.get("SFG_PARITY_RECORD")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(row) + "\n")


def check(config, quantity, got, dev32, f64, ref32=None):
    """Record and assert one row; f64 None: the FP32 comparison alone."""
    got = np.asarray(got, np.float64)
    assert np.all(np.isfinite(got))
    assert np.linalg.norm(dev32) > 0
    row = {"config": config, "quantity": quantity,
           "cuda_vs_oracle_f32_device_order": rel_l2(got, dev32)}
    if f64 is not None:
        assert np.linalg.norm(f64) > 0
        row["cuda_vs_oracle_f64"] = rel_l2(got, f64)
        row["oracle_f32_device_order_vs_f64"] = rel_l2(dev32, f64)
    if ref32 is not None:
        row["cuda_vs_oracle_f32_reference_order"] = rel_l2(got, ref32)
        row["oracle_f32_reference_order_vs_f64"] = rel_l2(ref32, f64)
    row["bound"] = bound(quantity, coupled=config.startswith("2 "))
    record(row)
    assert row["cuda_vs_oracle_f32_device_order"] <= row["bound"], row
    if ref32 is not None:
        assert row["cuda_vs_oracle_f32_reference_order"] <= row["bound"], row
    if f64 is not None:
        floor = max(row["oracle_f32_device_order_vs_f64"], row.get("oracle_f32_reference_order_vs_f64", 0.0))
        assert row["cuda_vs_oracle_f64"] <= 1.25 * floor + 1e-6, row


def run_cuda2d(w, srcs, nstep, types, nshots=1):
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=nstep, nshots=nshots, point_rho=w.point_rho,
                           point_vp=w.point_vp, point_vs=w.point_vs)
    sim.set_sources(srcs)
    sim.set_receivers(w.rec_x, w.rec_z, types=types)
    sim.initialize()
    sim.run(nstep)
    assert sim.check_finite()
    return sim


def oracle_runs(case, reference_order=True):
    from oracle import runner
    dev = oracle_f32(case, nthreads=NT, want_final=True)
    ref = runner.run(case, "f32", nthreads=NT, want_final=True) if reference_order else None
    r64 = runner.run(case, "f64", nthreads=NT, want_final=True)
    return dev, ref, r64


def elastic_points(sim, r, shot=None):
    """Final elastic displacement of the product and of oracle results r
    (dict of runs) at every element GLL point of the elastic medium."""
    ib_p, g2e, _ = sim.numbering()
    gl = ib_p.ravel()
    el = g2e[gl] >= 0
    u = sim.field("elastic", "displacement")
    if shot is not None:
        u = u[shot]
    ib_o = next(iter(v for v in r.values() if v is not None))["final"]["ibool"].ravel()
    return u[g2e[gl[el]]], {k: (v["final"]["elastic"][ib_o[el]] if v is not None else None) for k, v in r.items()}


def test_config1_elastic_80x60_full(sfg_lib, oracle_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=1600)
    types = ("displacement", "velocity", "acceleration")
    case = workload_case(w, types=types)
    dev, ref, r64 = oracle_runs(case)
    sim = run_cuda2d(w, w.sources, w.nstep, types)
    seis = sim.seismograms()[0]
    cfg = "1 elastic 80x60, 1600 steps"
    for t, kind in enumerate(types):
        check(cfg, kind, seis[:, t], dev["seis"][:, t], r64["seis"][:, t], ref["seis"][:, t])
    u, o = elastic_points(sim, {"dev": dev, "ref": ref, "f64": r64})
    check(cfg, "field:displacement", u, o["dev"], o["f64"], o["ref"])


def test_config2_coupled_400x200_full(sfg_lib, oracle_lib):
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200(nstep=4000)
    types = ("displacement", "velocity", "acceleration", "pressure")
    case = workload_case(w, types=types)
    dev, ref, r64 = oracle_runs(case)
    sim = run_cuda2d(w, w.sources, w.nstep, types)
    seis = sim.seismograms()[0]
    cfg = "2 coupled 400x200, 4000 steps"
    for t, kind in enumerate(types):
        check(cfg, kind, seis[:, t], dev["seis"][:, t], r64["seis"][:, t], ref["seis"][:, t])
    u, o = elastic_points(sim, {"dev": dev, "ref": ref, "f64": r64})
    check(cfg, "field:displacement (elastic)", u, o["dev"], o["f64"], o["ref"])
    ib_p, g2e, g2a = sim.numbering()
    gl = ib_p.ravel()
    ac = g2e[gl] < 0
    ib_o = dev["final"]["ibool"].ravel()[ac]
    chi = sim.field("acoustic", "displacement")[g2a[gl[ac]]]
    check(cfg, "field:potential (acoustic)", chi, dev["final"]["acoustic"][ib_o], r64["final"]["acoustic"][ib_o],
          ref["final"]["acoustic"][ib_o])


def test_config3_batched_1000x500_shots(sfg_lib, oracle_lib):
    from oracle import runner
    from specfempp_b200 import meshgen
    nstep = 300
    w = meshgen.elastic_grf_1000x500(nstep=nstep, nshots=32)
    types = ("displacement", "velocity")
    sim = run_cuda2d(w, w.sources, nstep, types, nshots=32)
    seis = sim.seismograms()               # [shot][nsig][ntypes][nrec][2]
    cfg = "3 batched 1000x500 GRF, 32 shots, 300 steps"
    for shot in (0, 15, 31):
        case = workload_case(w, nstep=nstep, types=types)
        case.sources = [replace(s, shot=0) for s in w.sources if s.shot == shot]
        dev = oracle_f32(case, nthreads=NT, want_final=True)
        # FP64 for shot 0 (the error statement); shots 15 and 31 against the
        # FP32 oracle alone (every shot runs the same arithmetic)
        r64 = runner.run(case, "f64", nthreads=NT, want_final=True) if shot == 0 else None
        u, o = elastic_points(sim, {"dev": dev, "f64": r64}, shot=shot)
        check(cfg, f"field:displacement, shot {shot}", u, o["dev"], o["f64"])
        if shot == 0:
            for t, kind in enumerate(types):
                check(cfg, f"{kind}:shot {shot}", seis[shot][:, t], dev["seis"][:, t], r64["seis"][:, t])


def test_config5_3d_128x128x64(sfg_lib, oracle_lib):
    from oracle import runner3d
    from specfempp_b200 import meshgen, sfg3d
    nstep = 60
    w = meshgen.elastic3d_layered_grf(128, 128, 64, nstep=nstep, nrec=1000)
    srcs = [replace(s, f0=10.0) for s in w.sources]
    sim = sfg3d.Simulation3D(w.mesh, dt=w.dt, nstep=nstep)
    sim.set_sources(srcs)
    sim.set_receivers(w.rec_xyz, types=("displacement",))
    sim.initialize()
    sim.run(nstep)
    assert sim.check_finite()
    u = sim.field("displacement")
    sim.close()
    case = runner3d.Case3D(w.mesh, srcs, w.rec_xyz, w.dt, nstep)
    dev = runner3d.run(replace(case, device_order=True), "f32", nthreads=NT, want_final=True)
    r64 = runner3d.run(case, "f64", nthreads=NT, want_final=True)
    check("5 3D 128x128x64, 60 steps", "field:displacement", u.ravel(), dev["final"].ravel(), r64["final"].ravel())
