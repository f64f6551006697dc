"""Edge cases of the 2D path against the oracle: no sources, no receivers,
sampling every n steps, rotated receivers, a source on a mesh node shared by
four elements and receivers on element edges, several sources in one
element; tolerances as in test_gpu_parity (1e-5 relative L2 for elastic
displacement and velocity)."""
from dataclasses import replace

import numpy as np
import pytest

from conftest import product_run, rel_l2, workload_case

pytestmark = pytest.mark.gpu


def elastic(nstep=500):
    from specfempp_b200 import meshgen
    return meshgen.elastic_psv_80x60(nstep=nstep)


def test_no_sources_stays_at_rest(sfg_lib):
    from specfempp_b200 import sfg
    w = elastic(100)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=100)
    sim.set_sources([])
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement", "velocity", "acceleration"))
    sim.initialize()
    sim.run(100)
    assert not np.any(sim.seismograms())
    assert not np.any(sim.field("elastic"))


def test_no_receivers(sfg_lib):
    from specfempp_b200 import sfg
    w = elastic(100)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=100)
    sim.set_sources(w.sources)
    sim.initialize()
    sim.run(100)
    assert sim.seismograms().size == 0
    assert np.abs(sim.field("elastic")).max() > 0


@pytest.mark.parametrize("nsb", [2, 7])
def test_sampling_every_n_steps(sfg_lib, oracle_lib, nsb):
    from oracle import runner
    w = elastic()
    case = workload_case(w, types=("displacement", "velocity"))
    case.nstep_between_samples = nsb
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    _, seis = product_run(case, types=case.seis_types)
    assert seis.shape[0] == (case.nstep + nsb - 1) // nsb
    for t in range(2):
        assert rel_l2(seis[:, t], ref[:, t]) <= 1e-5


def test_rotated_receivers(sfg_lib, oracle_lib):
    from oracle import runner
    w = elastic()
    case = workload_case(w, types=("displacement",))
    case.rec_angle = 30.0
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    _, seis = product_run(case, types=case.seis_types)
    assert rel_l2(seis, ref) <= 1e-5
    case.rec_angle = 0.0
    _, plain = product_run(case, types=case.seis_types)
    c, s = np.cos(np.pi / 6), np.sin(np.pi / 6)
    rot = np.stack([c * plain[..., 0] - s * plain[..., 1], s * plain[..., 0] + c * plain[..., 1]], -1)
    assert rel_l2(seis, rot) <= 1e-6


def test_source_on_node_receivers_on_edges_several_sources_per_element(sfg_lib, oracle_lib):
    from oracle import runner
    w = elastic()
    h = 4000.0 / 80
    s0 = w.sources[0]
    srcs = [replace(s0, x=40 * h, z=50 * h),                       # node shared by four elements
            replace(s0, x=30.2 * h, z=20.5 * h, factor=0.7 * s0.factor, angle=25.0),
            replace(s0, x=30.7 * h, z=20.3 * h, factor=-0.4 * s0.factor, f0=12.0)]   # same element
    case = workload_case(w, types=("displacement", "velocity"))
    case.sources = srcs
    case.rec_x = np.array([10 * h, 25.5 * h, 61 * h, 70 * h])
    case.rec_z = np.array([55.25 * h, 57 * h, 40 * h, 12 * h])               # on edges and a node
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    _, seis = product_run(case, types=case.seis_types)
    assert np.abs(ref).max() > 0
    for t in range(2):
        assert rel_l2(seis[:, t], ref[:, t]) <= 1e-5, (t, rel_l2(seis[:, t], ref[:, t]))
    # every element kernel gives the same bits with several sources per element
    _, base = product_run(case, types=case.seis_types, variant=1)
    for v in (2, 3, 4, 5, 6):
        _, s2 = product_run(case, types=case.seis_types, variant=v)
        assert np.array_equal(s2, base), v


TF_SPEC = [("ricker", 10.0, 0.0), ("dirac", 0.0, 0.0), ("gaussian", 12.0, 0.0), ("gaussian_hdur", 0.0, 0.02),
           ("dgaussian", 12.0, 0.0), ("heaviside", 0.0, 0.03)]


@pytest.mark.parametrize("which", list(range(len(TF_SPEC))) + ["all"],
                         ids=[k for k, _, _ in TF_SPEC] + ["all"])
def test_every_time_function_kind(sfg_lib, oracle_lib, which):
    """Sources with each time function (Ricker, Dirac, Gaussian by f0 and by
    hdur, dGaussian, Heaviside), each alone and all together (the earliest
    start sets everyone's time axis): the library's tables and run against the
    oracle's, displacement at 1e-5; velocity at max(1e-5, twice the oracle's
    own FP32-vs-FP64 difference), since the step-like time functions leave
    velocities whose FP32 rounding is larger (up to 5e-5 observed)."""
    from oracle import runner
    w = elastic(1400)
    s0 = w.sources[0]
    srcs = [runner.Source(x=600.0 + 550.0 * k, z=2300.0 + 60.0 * k, f0=f0, factor=s0.factor,
                          angle=15.0 * k, stf=kind, hdur=hdur)
            for k, (kind, f0, hdur) in enumerate(TF_SPEC)]
    case = workload_case(w, types=("displacement", "velocity"))
    case.sources = srcs if which == "all" else [srcs[which]]
    ref = runner.run(case, "f32", nthreads=8)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=case.seis_types)
    assert np.abs(ref).max() > 0
    for t in range(2):
        tol = 1e-5 if t == 0 else max(1e-5, 2.0 * rel_l2(ref[:, t], ref64[:, t]))
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (t, rel_l2(seis[:, t], ref[:, t]), tol)


def test_given_start_time(sfg_lib, oracle_lib):
    """A start time given by the caller (the configuration's t0): every
    source keeps its own tshift; seismograms against the oracle at 1e-5, the
    handle's t0 is the given one, and a start after the earliest source start
    is refused."""
    from oracle import runner
    from specfempp_b200 import sfg
    w = elastic(900)
    s0 = w.sources[0]
    srcs = [replace(s0, tshift=0.05), replace(s0, x=1200.0, z=2200.0, f0=14.0)]
    case = workload_case(w, types=("displacement", "velocity"))
    case.sources = srcs
    case.start_time = -0.2
    ref = runner.run(case, "f32", nthreads=8)["seis"]
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=900, start_time=-0.2)
    sim.set_sources(srcs)
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement", "velocity"))
    sim.initialize()
    sim.run(900)
    assert abs(sim.info().t0 - (-0.2)) < 1e-7
    seis = sim.seismograms()[0]
    for t in range(2):
        assert rel_l2(seis[:, t], ref[:, t]) <= 1e-5, (t, rel_l2(seis[:, t], ref[:, t]))
    late = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=900, start_time=-0.01)
    with pytest.raises(sfg.SfgError, match="start time"):
        late.set_sources(srcs)
