"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (fixed, relative L2, CUDA FP32 against oracle FP32), by medium of
the receivers and output; the bounds above 1e-5 sit on the FP32 noise floor
that the oracle itself shows (its FP32 run against its FP64 run, and two
FP32 runs that differ only in summation order):
* elastic displacement and velocity, final wavefields: 1e-5;
* elastic acceleration and pressure, Cosserat rotation and curl, and every
  output of coupled models (receivers in both media): 1e-4 (FP32 vs FP64
  2-5e-5);
* acoustic displacement (rho^-1 grad of the potential): 1e-4 (two summation
  orders differ by 1.3e-5);
* acoustic velocity, acceleration and pressure: 5e-3 (on the free-surface
  acoustic fixture FP32 vs FP64 is 9.5e-5, 1.4e-3 and 1.2e-4, two summation
  orders differ by 1.3e-4, 2.0e-3 and 1.8e-4);
* Cosserat intrinsic rotation (rotation minus half the curl, a
  cancellation): 5e-3 (FP32 vs FP64 7.7e-4);
* against the reference's golden traces: the reference's own metric
  sum|d|/sum|ref| per station < 1e-3 (newmark_tests.cpp:331-373).
The run is deterministic (colour-ordered assembly): two runs agree bitwise.
"""
import numpy as np
import pytest

from conftest import golden_case, product_run, reference_metric, rel_l2, workload_case

pytestmark = pytest.mark.gpu

FIXTURES = ["HomogeneousElasticDomain", "HomogeneousElasticDomainStaceyDirichletBC",
            "HomogeneousElasticDomainStaceyBC", "HomogeneousAcousticDomainDirichletBC",
            "AcousticElasticCoupledDomainVariant2", "HomogeneousElasticDomainMomentTensor",
            "HomogeneousElasticIsotropicDomainSH", "HomogeneousElasticAnisotropicDomain",
            "HomogeneousAcousticDomain", "HomogeneousAcousticDomainCompositeStaceyDirichletBC",
            "HomogeneousElasticDomainMomentTensorHeaviside", "HomogeneousElasticDomainWAdjacencyMap",
            "HomogeneousIsotropicCosseratDomainNu0", "AcousticElasticCoupledDomain"]


TOL_DV = 1e-5      # elastic displacement and velocity, final fields
TOL_AP = 1e-4      # elastic acceleration / pressure, rotation, curl, coupled models, acoustic displacement
TOL_NOISY = 5e-3   # acoustic velocity / acceleration / pressure, Cosserat intrinsic rotation


def tolerance(kind, f32=None, f64=None, medium="elastic"):
    """The fixed bound of an output (see the module docstring) for receivers
    in an elastic, acoustic or coupled model.  The FP32 and FP64 oracle
    results are accepted for the callers' convenience; the bound does not
    depend on them."""
    if kind == "intrinsic_rotation":
        return TOL_NOISY
    if medium == "acoustic":
        return TOL_AP if kind == "displacement" else TOL_NOISY
    if medium == "coupled":
        return TOL_AP
    return TOL_DV if kind in ("displacement", "velocity") else TOL_AP


@pytest.mark.parametrize("name", FIXTURES)
def test_golden_fixture_parity(sfg_lib, oracle_lib, name):
    from oracle import runner
    case, traces, _ = golden_case(name)
    ref = runner.run(case, "f32", nthreads=1)["seis"][:, 0]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"][:, 0]
    _, seis = product_run(case)
    got = seis[:, 0]
    assert np.all(np.isfinite(got))
    elastic = bool(np.all(case.mesh.mat_medium == 1))
    acoustic = bool(np.all(case.mesh.mat_medium == 0))
    tol = TOL_DV if elastic else tolerance("displacement", medium="acoustic" if acoustic else "coupled")
    assert rel_l2(got, ref) <= tol, (rel_l2(got, ref), tol)
    assert reference_metric(got, traces).max() < 1e-3


def test_elastic_psv_80x60_parity_and_fields(sfg_lib, oracle_lib):
    from oracle import runner
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=1000)
    case = workload_case(w, types=("displacement", "velocity", "acceleration"))
    r = runner.run(case, "f32", nthreads=1, want_final=True)
    r64 = runner.run(case, "f64", nthreads=8)
    sim, seis = product_run(case, types=case.seis_types)
    for t, kind in enumerate(case.seis_types):
        tol = 1e-5 if kind in ("displacement", "velocity") else tolerance(kind, r["seis"][:, t], r64["seis"][:, t])
        assert rel_l2(seis[:, t], r["seis"][:, t]) <= tol, (kind, rel_l2(seis[:, t], r["seis"][:, t]))
    # FP32 error against FP64, reported alongside (both builds)
    e_gpu = rel_l2(seis[:, 0], r64["seis"][:, 0])
    e_cpu = rel_l2(r["seis"][:, 0], r64["seis"][:, 0])
    assert e_gpu < 1e-4 and e_cpu < 1e-4
    # final displacement field through the two numberings
    ib_p, g2e, _ = sim.numbering()
    ib_o = r["final"]["ibool"]
    u_p = sim.field("elastic", "displacement")
    u_o = r["final"]["elastic"]
    mp = g2e[ib_p.ravel()]
    assert rel_l2(u_p[mp], u_o[ib_o.ravel()]) <= 1e-5


def test_coupled_small_parity(sfg_lib, oracle_lib):
    from oracle import runner
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200(nstep=600, nx=80, nz=40)
    types = ("displacement", "velocity", "acceleration", "pressure")
    case = workload_case(w, types=types)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=types)
    assert np.all(np.isfinite(seis))
    assert np.abs(ref[:, 0]).max() > 0
    for t, kind in enumerate(types):
        tol = tolerance(kind, medium="coupled")
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)


def test_acoustic_receivers_all_types(sfg_lib, oracle_lib):
    from oracle import runner
    case, _, _ = golden_case("HomogeneousAcousticDomainDirichletBC")
    types = ("displacement", "velocity", "acceleration", "pressure")
    case.seis_types = list(types)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=types)
    for t, kind in enumerate(types):
        tol = tolerance(kind, medium="acoustic")
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)


@pytest.mark.parametrize("epb,spg,variant", [(8, 7, 1), (32, 1, 1), (8, 3, 2), (16, 20, 2), (32, 5, 2),
                                             (8, 4, 3), (16, 20, 3), (32, 1, 3),
                                             (8, 4, 4), (16, 20, 4), (32, 1, 4),
                                             (16, 20, 5), (16, 3, 5), (16, 1, 5),
                                             (32, 20, 6), (16, 3, 6), (32, 1, 6)])
def test_launch_shapes_and_graphs_agree(sfg_lib, epb, spg, variant):
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200(nstep=120, nx=40, nz=20)
    case = workload_case(w)
    _, a = product_run(case, epb=16, variant=1)
    _, b = product_run(case, epb=epb, spg=spg, variant=variant)
    # a different block shape or element order inside a colour changes no
    # summation order: bitwise equal
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())


def test_deterministic(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=200)
    case = workload_case(w)
    sim, a = product_run(case)
    sim.reset()
    sim.run(case.nstep)
    b = sim.seismograms()[0]
    assert np.array_equal(a, b)
    assert sim.check_finite()


def test_fields_after_timing_call_are_refused(sfg_lib):
    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=20)
    sim, _ = product_run(workload_case(w))
    sim.field("elastic")
    sim.run_timed_flushed(3, 1 << 20)
    with pytest.raises(sfg.SfgError) as e:
        sim.field("elastic")
    assert e.value.code == -5
    sim.run(1)
    assert np.all(np.isfinite(sim.field("elastic")))


def test_kernel_timing_with_flushed_cache(sfg_lib):
    """sfg_time_kernel_flushed: every launch after an L2 flush; its inputs come
    from HBM, so it takes at least about as long as back to back."""
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200(nstep=20, nx=200, nz=100)
    sim, _ = product_run(workload_case(w), nsteps=5)
    b2b = sim.time_kernel(0, 10)
    cold = sim.time_kernel(0, 10, 256 << 20)
    assert b2b > 0 and cold > 0
    assert cold >= 0.8 * b2b, (cold, b2b)
    sim.reset()
    sim.run(3)
    assert sim.check_finite()


def test_step_and_run_agree(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=50)
    case = workload_case(w)
    sim, a = product_run(case)
    sim.reset()
    for _ in range(case.nstep):
        sim.step()
    assert np.array_equal(a, sim.seismograms()[0])


@pytest.mark.parametrize("name", ["HomogeneousAcousticDomainDirichletBC", "HomogeneousElasticDomainStaceyBC",
                                  "HomogeneousElasticIsotropicDomainSH", "HomogeneousElasticDomainMomentTensor"])
@pytest.mark.parametrize("variant", [3, 4, 5, 6])
def test_owner_computes_variants_equal_colour_passes(sfg_lib, name, variant):
    """Single-medium fixtures: the owner-computes kernels (plain, with
    bulk-copy staging, fused tiles and the row form; media a form does not
    cover fall back to plain owner-computes) give the colour passes' bits."""
    case, _, _ = golden_case(name)
    _, a = product_run(case, epb=16, variant=1)
    _, b = product_run(case, epb=8, variant=variant)
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())


@pytest.mark.parametrize("name", ["HomogeneousElasticDomainMomentTensor", "HomogeneousElasticIsotropicDomainSH",
                                  "HomogeneousElasticAnisotropicDomain"])
def test_moment_tensor_and_sh_all_types(sfg_lib, oracle_lib, name):
    """Moment-tensor source (P-SV) and SH: displacement, velocity and
    acceleration against the oracle (tolerances above) and against the
    reference's golden traces (sum|d|/sum|ref| < 1e-3)."""
    import os
    from conftest import GOLDEN
    from oracle import runner
    case, _, _ = golden_case(name)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    types = ("displacement", "velocity", "acceleration")
    case.seis_types = list(types)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    _, seis = product_run(case, types=types)
    for t, (kind, key) in enumerate(zip(types, ("traces", "traces_semv", "traces_sema"))):
        tol = 1e-5 if kind == "displacement" else tolerance(kind, ref[:, t], ref64[:, t])
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)
        assert reference_metric(seis[:, t], z[key]).max() < 1e-3, kind


def test_step_io_matches_run(sfg_lib):
    """The per-step host-buffer path gives the run's seismograms bit for bit
    (with the library's own source table and with the same table streamed in
    from the host); its fields are mid-step until a plain step ends the run."""
    from specfempp_b200 import meshgen, sfg, stf
    w = meshgen.elastic_psv_80x60(nstep=60)
    case = workload_case(w)
    sim, a = product_run(case)
    inf = sim.info()
    table = stf.table(w.sources, w.dt, case.nstep).astype(np.float32)
    for streamed in (False, True):
        sim.reset()
        row = np.zeros((inf.nshots, inf.ntypes, inf.nrec, 2), np.float32)
        rows = []
        for k in range(case.nstep - 1):
            sim.step_io(np.ascontiguousarray(table[k]) if streamed else None, row)
            rows.append(row[0].copy())
        with pytest.raises(sfg.SfgError):
            sim.field("elastic")
        sim.step()
        got = np.concatenate([np.stack(rows), sim.seismograms()[0][-1:]])
        if streamed:
            assert np.allclose(got, a, rtol=0, atol=1e-6 * np.abs(a).max())
        else:
            assert np.array_equal(got, a)
        assert np.all(np.isfinite(sim.field("elastic")))


def test_anisotropic_layered_parity(sfg_lib, oracle_lib):
    """Tilted anisotropic half (c15, c35 != 0) under an isotropic half, Stacey
    on three sides: displacement and velocity against the oracle at 1e-5,
    acceleration at the FP32 noise tolerance; the owner-computes kernel gives
    the colour passes' bits."""
    from oracle import runner
    from test_oracle import layered_aniso_case
    case = layered_aniso_case(1200)
    types = ("displacement", "velocity", "acceleration")
    case.seis_types = list(types)
    ref = runner.run(case, "f32", nthreads=1)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    sim, seis = product_run(case, types=types, variant=1)
    assert sim.info().kernel_variant == 1
    for t, kind in enumerate(types):
        tol = 1e-5 if kind != "acceleration" else tolerance(kind, ref[:, t], ref64[:, t])
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)
    for v in (0, 2, 3, 4, 5, 6):
        _, s2 = product_run(case, types=types, variant=v)
        assert np.array_equal(s2, seis), v


def test_anisotropic_unsupported_forms(sfg_lib):
    """The anisotropic medium is P-SV only: elastic pressure seismograms, SH,
    batched shots and the adjoint are refused with SFG_ERR_UNSUPPORTED."""
    from specfempp_b200 import sfg
    from test_oracle import layered_aniso_case
    case = layered_aniso_case(10)
    sim = sfg.Simulation2D(case.mesh, dt=case.dt, nstep=10)
    sim.set_sources(case.sources)
    sim.set_receivers(case.rec_x, case.rec_z, 0.0, ("pressure",))
    with pytest.raises(sfg.SfgError, match="isotropic"):
        sim.initialize()
    with pytest.raises(sfg.SfgError):
        sfg.Simulation2D(case.mesh, dt=case.dt, nstep=10, elastic_wave="sh")
    with pytest.raises(sfg.SfgError):
        sfg.Simulation2D(case.mesh, dt=case.dt, nstep=10, nshots=4)


COSSERAT = {
    "HomogeneousIsotropicCosseratDomain": ["displacement", "rotation", "intrinsic_rotation", "curl", "pressure"],
    "HomogeneousIsotropicCosseratDomainHighFrequency": ["displacement", "velocity", "rotation", "curl"],
    "cosserat_80x60_stacey": ["displacement", "velocity", "acceleration", "rotation", "intrinsic_rotation",
                              "curl", "pressure"],
}


@pytest.mark.parametrize("name", list(COSSERAT))
def test_cosserat_parity(sfg_lib, oracle_lib, name):
    """Isotropic Cosserat P-SV-T fixtures (displacement + rotation, couple
    stress): every seismogram type against the oracle at the fixed bounds of
    its class (module docstring); colour passes and owner-computes give the
    same bits."""
    from oracle import runner
    if name == "cosserat_80x60_stacey":
        from test_oracle import cosserat_80x60
        case = cosserat_80x60(1200)
    else:
        case, _, _ = golden_case(name)
    types = COSSERAT[name]
    case.seis_types = list(types)
    ref = runner.run(case, "f32", nthreads=8)["seis"]
    ref64 = runner.run(case, "f64", nthreads=8)["seis"]
    sim, seis = product_run(case, types=types, variant=1)
    assert sim.info().ncomp_elastic == 3
    for t, kind in enumerate(types):
        tol = 1e-5 if kind == "displacement" else tolerance(kind, ref[:, t], ref64[:, t])
        assert rel_l2(seis[:, t], ref[:, t]) <= tol, (kind, rel_l2(seis[:, t], ref[:, t]), tol)
    _, s3 = product_run(case, types=types, variant=3)
    assert np.array_equal(s3, seis)
