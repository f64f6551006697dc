"""The fused tile kernel (kernel variant 5) against the other variants.

Variant 5 computes element forces, assembles them in shared memory tile by
tile and finishes the tile-interior points in one launch; a second launch
finishes the points that tiles share (and the coupled interface), a third
interpolates the receivers from the end-of-step values of their points.
Every point's contributions are still summed in colour order, so its
seismograms and fields must equal the colour-pass kernel's bit for bit, for
every seismogram type, with sources, Stacey edges, free surfaces and the
acoustic-elastic coupling, across runs cut into pieces, single steps and the
per-step host-buffer call.
"""
import numpy as np
import pytest

from conftest import golden_case, product_run, workload_case

pytestmark = pytest.mark.gpu

ALL_TYPES = ("displacement", "velocity", "acceleration", "pressure")


def _fields(sim):
    out = {}
    inf = sim.info()
    for med, n in (("elastic", inf.nglob_elastic), ("acoustic", inf.nglob_acoustic)):
        if n == 0:
            continue
        for f in ("displacement", "velocity", "acceleration"):
            out[(med, f)] = sim.field(med, f)
    return out


def _equal_runs(case, types, nsteps=None):
    s1, a = product_run(case, types=types, nsteps=nsteps, variant=1)
    s5, b = product_run(case, types=types, nsteps=nsteps, variant=5)
    assert s5.info().kernel_variant == 5
    assert s5.info().kernels_per_step <= 4
    assert np.abs(a).max() > 0
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())
    fa, fb = _fields(s1), _fields(s5)
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k
    assert s5.check_finite()
    return s5


@pytest.mark.parametrize("nx,nz", [(40, 20), (80, 40)])
def test_tile_kernel_coupled_all_types(sfg_lib, nx, nz):
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200(nstep=150, nx=nx, nz=nz)
    case = workload_case(w, types=ALL_TYPES)
    _equal_runs(case, ALL_TYPES)


@pytest.mark.parametrize("name", ["HomogeneousAcousticDomainDirichletBC", "HomogeneousElasticDomainStaceyBC",
                                  "HomogeneousElasticDomainStaceyDirichletBC",
                                  "HomogeneousElasticIsotropicDomainSH", "HomogeneousElasticDomainMomentTensor",
                                  "AcousticElasticCoupledDomainVariant2", "HomogeneousAcousticDomain",
                                  "HomogeneousAcousticDomainCompositeStaceyDirichletBC"])
def test_tile_kernel_fixtures(sfg_lib, name):
    case, _, _ = golden_case(name)
    types = ALL_TYPES if not case.elastic_sh else ("displacement", "velocity", "acceleration")
    _equal_runs(case, types, nsteps=min(case.nstep, 800))


def test_tile_kernel_elastic_80x60(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=400)
    _equal_runs(workload_case(w, types=ALL_TYPES), ALL_TYPES)


def test_tile_kernel_pieces_steps_and_step_io(sfg_lib):
    """Runs cut into pieces, single steps and the host-buffer step give the
    one-run seismograms (the pending predictor is resumed between runs)."""
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200(nstep=90, nx=40, nz=20)
    case = workload_case(w, types=("displacement", "velocity"))
    sim, whole = product_run(case, types=case.seis_types, variant=5)
    sim.reset()
    sim.run(37)
    for _ in range(3):
        sim.step()
    sim.run(50)
    assert np.array_equal(sim.seismograms()[0], whole)
    sim.reset()
    inf = sim.info()
    got = np.zeros((case.nstep, inf.ntypes, inf.nrec, 2), np.float32)
    row = np.zeros((inf.nshots, inf.ntypes, inf.nrec, 2), np.float32)
    for i in range(case.nstep):
        sim.step_io(None, row)
        got[i] = row[0]
    assert np.array_equal(got, whole)


def test_tile_kernel_new_sources_and_model(sfg_lib):
    """Replacing the sources and the model after initialisation refreshes the
    tile records: the results equal a handle built with them."""
    from dataclasses import replace

    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=200)
    src2 = [replace(w.sources[0], x=w.sources[0].x + 700.0, z=w.sources[0].z - 400.0)]

    def make(srcs):
        sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep, kernel_variant=5)
        sim.set_sources(srcs)
        sim.set_receivers(w.rec_x, w.rec_z, types=("displacement", "velocity"))
        sim.initialize()
        return sim

    a = make(w.sources)
    a.set_sources(src2)
    a.run(w.nstep)
    b = make(src2)
    b.run(w.nstep)
    assert a.info().kernel_variant == 5
    assert np.array_equal(a.seismograms(), b.seismograms())
    # model: 3% slower shear waves everywhere, against the colour passes
    nspec = w.mesh.nspec
    rho = np.full((nspec, 25), float(w.mesh.mat_rho[0]), np.float32)
    vp = float(w.mesh.mat_vp[0])
    vs = 0.97 * float(w.mesh.mat_vs[0])
    mu = rho * vs * vs
    kappa = rho * vp * vp - 4.0 / 3.0 * mu
    out = []
    for v in (1, 5):
        sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep, kernel_variant=v)
        sim.set_sources(w.sources)
        sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
        sim.initialize()
        sim.set_model(rho, kappa.astype(np.float32), mu.astype(np.float32))
        sim.run(w.nstep)
        out.append(sim.seismograms())
    assert np.array_equal(out[0], out[1])


def test_tile_kernel_refused_forms_fall_back(sfg_lib):
    """Models the tile kernel does not cover (anisotropic) run another
    variant when variant 5 is asked for."""
    from test_oracle import layered_aniso_case
    case = layered_aniso_case(50)
    sim, _ = product_run(case, variant=5)
    assert sim.info().kernel_variant == 3


# ---------------------------------------------------------------------------
# Batched shots (S a multiple of 4): the same tiles, one work item per tile
# and quad of shots; every shot's bits must equal the colour-pass run's.

def _batched_shots(nshots, seed, xr, zr):
    from specfempp_b200 import meshgen
    rng = np.random.default_rng(seed)
    return [meshgen.RickerSource(float(rng.uniform(*xr)), float(rng.uniform(*zr)), float(rng.uniform(6.0, 14.0)),
                                 1e10, shot=s) for s in range(nshots)]


def _batched_run(case, srcs, nshots, types, variant, pieces=(None,)):
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(case.mesh, dt=case.dt, nstep=case.nstep, nshots=nshots,
                           elastic_wave="sh" if case.elastic_sh else "psv",
                           point_rho=case.point_rho, point_vp=case.point_vp, point_vs=case.point_vs,
                           kernel_variant=variant)
    sim.set_sources(srcs)
    sim.set_receivers(case.rec_x, case.rec_z, case.rec_angle, types)
    sim.initialize()
    for n in pieces:
        sim.run(case.nstep if n is None else n)
    return sim


def _batched_equal(case, srcs, nshots, types, pieces=(None,)):
    s1 = _batched_run(case, srcs, nshots, types, 1)
    s5 = _batched_run(case, srcs, nshots, types, 5, pieces)
    assert s5.info().kernel_variant == 5
    a, b = s1.seismograms(), s5.seismograms()
    assert a.shape[0] == nshots and np.abs(a).max() > 0
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())
    for f in ("displacement", "velocity", "acceleration"):
        fa, fb = s1.field("elastic", f), s5.field("elastic", f)
        assert np.abs(fa).max() > 0
        assert np.array_equal(fa, fb), f
    assert s5.check_finite()


@pytest.mark.parametrize("nshots", [4, 8, 12])
def test_batched_tile_kernel_elastic_80x60(sfg_lib, nshots):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=300)
    case = workload_case(w)
    types = ("displacement", "velocity", "acceleration")
    _batched_equal(case, _batched_shots(nshots, 5, (600, 3400), (600, 2600)), nshots, types)


def test_batched_tile_kernel_grf_model_in_pieces(sfg_lib):
    """Heterogeneous model, a run cut into pieces (the pending predictor is
    resumed between runs)."""
    from specfempp_b200 import meshgen
    w = meshgen.elastic_grf_1000x500(nstep=120, nshots=8, nx=100, nz=50)
    case = workload_case(w)
    types = ("displacement", "velocity", "acceleration")
    _batched_equal(case, w.sources, 8, types, pieces=(50, 1, 69))


@pytest.mark.parametrize("name", ["HomogeneousElasticDomainStaceyDirichletBC", "HomogeneousElasticIsotropicDomainSH"])
def test_batched_tile_kernel_fixtures(sfg_lib, name):
    case, _, _ = golden_case(name)
    case.nstep = min(case.nstep, 600)
    xs = [float(x) for x in case.rec_x]
    zs = [float(z) for z in case.rec_z]
    srcs = _batched_shots(8, 11, (min(xs), max(xs)), (min(zs), max(zs)))
    _batched_equal(case, srcs, 8, ("displacement", "velocity", "acceleration"))


# ---------------------------------------------------------------------------
# Batched tiles of four elements (variant 7): tile-interior points assembled
# and finished in the tile kernel, shared points by the list update;
# displacement receivers.

def _btile_equal(case, srcs, nshots, pieces=(None,)):
    types = ("displacement",)
    s1 = _batched_run(case, srcs, nshots, types, 1)
    s7 = _batched_run(case, srcs, nshots, types, 7, pieces)
    assert s7.info().kernel_variant == 7
    a, b = s1.seismograms(), s7.seismograms()
    assert np.abs(a).max() > 0
    assert np.array_equal(a, b), float(np.abs(a - b).max() / np.abs(a).max())
    for f in ("displacement", "velocity", "acceleration"):
        fa, fb = s1.field("elastic", f), s7.field("elastic", f)
        assert np.abs(fa).max() > 0
        assert np.array_equal(fa, fb), f
    assert s7.check_finite()


@pytest.mark.parametrize("nshots", [4, 8, 36])
def test_batched_four_element_tiles_elastic_80x60(sfg_lib, nshots):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=300)
    _btile_equal(workload_case(w), _batched_shots(nshots, 5, (600, 3400), (600, 2600)), nshots)


def test_batched_four_element_tiles_grf_in_pieces(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_grf_1000x500(nstep=120, nshots=8, nx=100, nz=50)
    _btile_equal(workload_case(w), w.sources, 8, pieces=(50, 1, 69))


@pytest.mark.parametrize("name", ["HomogeneousElasticDomainStaceyDirichletBC", "HomogeneousElasticIsotropicDomainSH"])
def test_batched_four_element_tiles_fixtures(sfg_lib, name):
    case, _, _ = golden_case(name)
    case.nstep = min(case.nstep, 600)
    xs = [float(x) for x in case.rec_x]
    zs = [float(z) for z in case.rec_z]
    _btile_equal(case, _batched_shots(8, 11, (min(xs), max(xs)), (min(zs), max(zs))), 8)
