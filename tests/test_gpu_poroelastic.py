"""Isotropic poroelastic medium on the CUDA path, against the oracle.

Tolerances as in test_gpu_parity: relative L2 <= max(1e-5, 2 x the oracle's
own FP32-vs-FP64 gap) against the oracle's FP32 run; the reference's golden
traces of its poroelastic fixture with its metric and tolerance 1e-3.  The
CUDA path folds the phase factors (1 - phi/tort, 1 - rho_f/rho_bar) into the
source arrays at setup, the oracle applies them per step as the reference
does: the two agree to FP32 rounding, not bitwise.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_case, product_run, reference_metric, rel_l2, workload_case
from test_gpu_parity import tolerance

pytestmark = pytest.mark.gpu

TYPES = ("displacement", "velocity", "acceleration", "pressure")


def test_poroelastic_golden_parity(sfg_lib, oracle_lib):
    from oracle import runner
    case, traces, _ = golden_case("PoroelasticCoupledDomainPSV")
    z = np.load(os.path.join(GOLDEN, "PoroelasticCoupledDomainPSV.npz"))
    case.seis_types = list(TYPES)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    sim, seis = product_run(case, types=TYPES)
    assert sim.info().ncomp_elastic == 4
    assert np.all(np.isfinite(seis))
    for t, kind in enumerate(TYPES):
        tol = tolerance(kind, ref[:, t], ref64[:, t])
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)
    for t, key in enumerate(("traces", "traces_semv", "traces_sema")):
        assert reference_metric(seis[:, t], z[key]).max() < 1e-3, key


def test_poroelastic_viscous_layered_parity(sfg_lib, oracle_lib):
    """Two porous layers, a viscous pore fluid with an anisotropic
    permeability (kxz != 0): the damping path against the oracle."""
    from oracle import runner
    from specfempp_b200 import meshgen
    w = meshgen.poroelastic_model(nx=40, nz=40, eta_f=1e-3, kxz=2e-10, nstep=800, layered=True)
    case = workload_case(w, types=TYPES)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=TYPES)
    assert np.abs(ref[:, 0]).max() > 0
    for t, kind in enumerate(TYPES):
        tol = tolerance(kind, ref[:, t], ref64[:, t])
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)


@pytest.mark.parametrize("epb,spg,variant", [(8, 7, 1), (32, 1, 1), (16, 3, 2), (8, 4, 3), (32, 5, 3),
                                             (16, 20, 4)])
def test_poroelastic_launch_shapes_agree(sfg_lib, epb, spg, variant):
    """Colour passes and owner-computes (the persistent and bulk-copy
    variants map to them) give the same bits for every block shape."""
    from specfempp_b200 import meshgen
    w = meshgen.poroelastic_model(nx=30, nz=30, eta_f=1e-3, nstep=200, layered=True)
    case = workload_case(w, types=("displacement", "pressure"))
    _, a = product_run(case, types=case.seis_types, epb=16, variant=1)
    _, b = product_run(case, types=case.seis_types, epb=epb, spg=spg, variant=variant)
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())


def test_poroelastic_database_front_end(sfg_lib, tmp_path):
    """The model written as a database.bin (material type 3) and read by the
    product's reader gives the in-memory run's bits."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.poroelastic_model(nx=30, nz=30, eta_f=1e-3, nstep=300, layered=True)
    case = workload_case(w)
    _, a = product_run(case)
    path = str(tmp_path / "database.bin")
    meshgen.write_database(w.mesh, path)
    sim = sfg.Simulation2D(database=path, dt=case.dt, nstep=case.nstep)
    sim.set_sources(case.sources)
    sim.set_receivers(case.rec_x, case.rec_z, case.rec_angle, ("displacement",))
    sim.initialize()
    sim.run(case.nstep)
    assert np.array_equal(a, sim.seismograms()[0])


def test_poroelastic_fields_and_refusals(sfg_lib):
    """The four-component fields come back in the handle's numbering; the
    adjoint and batched shots refuse the medium."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.poroelastic_model(nx=12, nz=12, nstep=50)
    sim, _ = product_run(workload_case(w))
    u = sim.field("elastic", "displacement")
    assert u.shape[1] == 4 and np.all(np.isfinite(u)) and np.abs(u[:, 2:]).max() > 0
    with pytest.raises(sfg.SfgError):
        sim.forward_checkpointed(10, 5)
    with pytest.raises(sfg.SfgError, match="batched"):
        sfg.Simulation2D(w.mesh, dt=w.dt, nstep=10, nshots=2)
