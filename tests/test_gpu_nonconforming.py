"""Nonconforming acoustic-elastic coupling on the CUDA path, against the oracle.

Tolerances as in test_gpu_parity: relative L2 <= max(1e-5, 2 x the oracle's
own FP32-vs-FP64 gap) against the oracle's FP32 run; the reference's golden
traces of its nonconforming fixture with its metric and tolerance 1e-2
(config.yaml of AcousticElasticNonconformingCoupledDomain).  The CUDA path
applies each interface point's coupling as one weighted sum over the other
medium's points (the intersection quadrature folded into per-pair weights
at setup), the oracle per quadrature point as the reference does: the two
agree to FP32 rounding, not bitwise.
"""
import numpy as np
import pytest

from conftest import golden_case, product_run, reference_metric, rel_l2, workload_case
from test_gpu_parity import tolerance

pytestmark = pytest.mark.gpu

TYPES = ("displacement", "velocity", "acceleration", "pressure")


def test_nonconforming_golden_parity(sfg_lib, oracle_lib):
    from oracle import runner
    case, traces, _ = golden_case("AcousticElasticNonconformingCoupledDomain")
    case.seis_types = list(TYPES)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=TYPES)
    assert np.all(np.isfinite(seis))
    assert np.abs(seis[:, 0, :2]).max() > 0               # elastic receivers, reached through the interface
    for t, kind in enumerate(TYPES):
        tol = tolerance(kind, medium="coupled")
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)
    assert reference_metric(seis[:, 0], traces).max() < 1e-2


def test_nonconforming_synthetic_parity(sfg_lib, oracle_lib):
    """30 elastic columns under 45 water columns (each elastic interface edge
    meets two or three water edges), Stacey sides, free surface on top."""
    from oracle import runner
    from specfempp_b200 import meshgen
    w = meshgen.nonconforming_coupled(nstep=1200)
    case = workload_case(w, types=TYPES)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=TYPES)
    assert np.abs(ref[:, 0, :4]).max() > 0
    for t, kind in enumerate(TYPES):
        tol = tolerance(kind, medium="coupled")
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)


def test_nonconforming_coincident_edges_match_conforming_twin(sfg_lib):
    """Coincident interface edges listed as nonconforming records give the
    run of the conforming twin that shares the interface nodes."""
    from specfempp_b200 import meshgen
    w = meshgen.nonconforming_coupled(nx_el=30, nx_ac=30, nstep=1200)
    _, a = product_run(workload_case(w))
    w.mesh = meshgen.merge_interface_nodes(w.mesh)
    _, b = product_run(workload_case(w))
    assert np.abs(b[:, 0, :4]).max() > 0
    assert rel_l2(a, b) <= 1e-5, rel_l2(a, b)


@pytest.mark.parametrize("epb,spg,variant", [(8, 7, 1), (16, 3, 2), (32, 5, 3), (16, 20, 4)])
def test_nonconforming_launch_shapes_agree(sfg_lib, epb, spg, variant):
    """Every kernel variant, block shape and graph length gives the same bits."""
    from specfempp_b200 import meshgen
    w = meshgen.nonconforming_coupled(nstep=200)
    case = workload_case(w)
    _, a = product_run(case, epb=16, variant=1)
    _, b = product_run(case, epb=epb, spg=spg, variant=variant)
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())


def test_nonconforming_database_front_end(sfg_lib, tmp_path):
    """The same mesh written as a database.bin with its adjacency records and
    read by the product's database reader gives the in-memory run's bits."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.nonconforming_coupled(nstep=300)
    case = workload_case(w)
    _, a = product_run(case)
    path = str(tmp_path / "database.bin")
    meshgen.write_database(w.mesh, path)
    sim = sfg.Simulation2D(database=path, dt=case.dt, nstep=case.nstep)
    sim.set_sources(case.sources)
    sim.set_receivers(case.rec_x, case.rec_z, case.rec_angle, ("displacement",))
    sim.initialize()
    sim.run(case.nstep)
    b = sim.seismograms()[0]
    assert np.array_equal(a, b)

