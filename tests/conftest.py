"""Shared test helpers.

Tests marked ``gpu`` need a CUDA device and the built libsfg.so; everything
else runs on CPU (oracle against the golden fixtures, the host-side
assembly and the C ABI's symbol table).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and libsfg.so")


def golden_case(name, nstep=None):
    """Rebuild an oracle Case2D (and golden traces) from tests/golden/<name>.npz."""
    from oracle import runner
    from oracle.database2d import Mesh2D

    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    mesh = Mesh2D(nspec=int(z["nspec"]), npgeo=int(z["npgeo"]), ngnod=int(z["ngnod"]),
                  coorg=z["coorg"], knods=z["knods"], kmato=z["kmato"],
                  mat_medium=z["mat_medium"], mat_rho=z["mat_rho"], mat_vp=z["mat_vp"],
                  mat_vs=z["mat_vs"], abs_ispec=z["abs_ispec"], abs_type=z["abs_type"],
                  free_ispec=z["free_ispec"], free_type=z["free_type"],
                  coupled_pairs=np.zeros((0, 2), np.int32),
                  mat_aniso=z["mat_aniso"] if "mat_aniso" in z else None,
                  mat_cosserat=z["mat_cosserat"] if "mat_cosserat" in z else None,
                  mat_poro=z["mat_poro"] if "mat_poro" in z else None)
    if "adjacency" in z:
        mesh.extra["adjacency"] = z["adjacency"]
    srcs = []
    for s in z["src"]:
        mt = len(s) > 7 and bool(s[7])
        codes = ["ricker", "dirac", "gaussian", "gaussian_hdur", "dgaussian", "heaviside"]
        stf = codes[int(s[11])] if len(s) > 11 else ("dirac" if s[6] else "ricker")
        srcs.append(runner.Source(x=s[0], z=s[1], f0=s[2], factor=s[3], tshift=s[4], angle=s[5],
                                  stf=stf, hdur=float(s[12]) if len(s) > 12 else 0.0,
                                  kind="moment_tensor" if mt else "force",
                                  mxx=s[8] if mt else 0.0, mzz=s[9] if mt else 0.0, mxz=s[10] if mt else 0.0))
    case = runner.Case2D(mesh=mesh, sources=srcs, rec_x=z["rec_x"], rec_z=z["rec_z"],
                         dt=float(z["dt"]), nstep=int(nstep or z["nstep"]),
                         rec_angle=float(z["rec_angle"]),
                         elastic_sh=bool(int(z["elastic_sh"])) if "elastic_sh" in z else False)
    return case, z["traces"], float(z["trace_t0"])


def reference_metric(computed, traces):
    """Per-station sum|d|/sum|ref| over components (newmark_tests.cpp:331-373).

    computed: [nsig, nrec, ncomp]; traces: [nrec, ncomp, nsig]."""
    n = min(computed.shape[0], traces.shape[2])
    c = np.transpose(computed[:n, :, :traces.shape[1]], (1, 2, 0))
    t = traces[:, :, :n]
    return np.abs(c - t).sum(axis=(1, 2)) / np.abs(t).sum(axis=(1, 2))


def oracle_f32(case, nthreads=8, want_final=False):
    """FP32 oracle run in the device kernels' evaluation order: the same
    algorithm as the reference-order oracle (which tests/test_oracle.py pins
    to the reference's golden traces), with the 5-term contractions as fused
    multiply-adds and the divergence weights hprime * w rounded once, as the
    CUDA kernels compute them.  The checker of the CUDA path: with the
    evaluation order shared, the two agree to FP32 round-off at any size,
    where the reference-order FP32 run differs from both by its own rounding
    (up to 5e-5 in long-run velocity and acceleration, as far from FP64 as
    the device order is)."""
    from dataclasses import replace

    from oracle import runner
    return runner.run(replace(case, device_order=True), "f32", nthreads=nthreads, want_final=want_final)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import runner
    runner.build()
    return runner.lib()


@pytest.fixture(scope="session")
def sfg_lib():
    from specfempp_b200 import build, sfg
    build.build()
    return sfg.load_library()


def product_run(case, types=("displacement",), nsteps=None, epb=0, spg=0, variant=0):
    """Run the CUDA path (libsfg through the C ABI) on an oracle Case2D."""
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(case.mesh, dt=case.dt, nstep=case.nstep,
                           nstep_between_samples=case.nstep_between_samples,
                           elastic_wave="sh" if case.elastic_sh else "psv",
                           point_rho=case.point_rho, point_vp=case.point_vp, point_vs=case.point_vs,
                           elements_per_block=epb, steps_per_graph=spg, kernel_variant=variant)
    sim.set_sources(case.sources)
    sim.set_receivers(case.rec_x, case.rec_z, case.rec_angle, types)
    sim.initialize()
    sim.run(case.nstep if nsteps is None else nsteps)
    seis = sim.seismograms()[0]
    return sim, seis


def workload_case(w, nstep=None, types=("displacement",)):
    """oracle Case2D of a meshgen Workload."""
    from oracle import runner
    return runner.Case2D(mesh=w.mesh, sources=w.sources, rec_x=w.rec_x, rec_z=w.rec_z, dt=w.dt,
                         nstep=int(nstep or w.nstep), seis_types=list(types),
                         point_rho=w.point_rho, point_vp=w.point_vp, point_vs=w.point_vs)
