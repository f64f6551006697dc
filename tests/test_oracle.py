"""The CPU oracle against the reference's golden vectors (CPU only).

Pins the oracle before it is used as the checker of the CUDA path:
* end-to-end traces of SPECFEM++'s Newmark regression fixtures (produced by
  Fortran SPECFEM2D), with the reference's own metric and tolerance 1e-3
  (tests/unit-tests/displacement_tests/Newmark/dim2/newmark_tests.cpp:331-373);
* known-answer tests from tests/unit-tests/gll/gll_tests.cpp and
  tests/unit-tests/medium/stress/dim2/elastic_isotropic.cpp.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_case, reference_metric

FIXTURES = ["HomogeneousElasticDomain", "HomogeneousElasticDomainStaceyDirichletBC",
            "HomogeneousElasticDomainStaceyBC", "HomogeneousAcousticDomainDirichletBC",
            "AcousticElasticCoupledDomainVariant2", "HomogeneousElasticDomainMomentTensor",
            "HomogeneousElasticIsotropicDomainSH", "HomogeneousElasticAnisotropicDomain",
            "HomogeneousAcousticDomain", "HomogeneousAcousticDomainCompositeStaceyDirichletBC",
            "HomogeneousElasticDomainMomentTensorHeaviside", "HomogeneousElasticDomainWAdjacencyMap",
            "AcousticElasticCoupledDomain"]


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_matches_golden_traces(oracle_lib, name):
    from oracle import runner
    case, traces, t0 = golden_case(name)
    r = runner.run(case, "f32", nthreads=8)
    assert abs(r["t0"] - t0) < 1e-3                     # time axis alignment
    err = reference_metric(r["seis"][:, 0], traces)
    assert np.all(np.isfinite(err))
    assert err.max() < 1e-3, err                          # the reference's tolerance
    assert err.max() < 5e-4                               # observed margin: <= 2e-4


@pytest.mark.parametrize("name", ["HomogeneousElasticDomainMomentTensor", "HomogeneousElasticIsotropicDomainSH",
                                  "HomogeneousElasticAnisotropicDomain"])
@pytest.mark.parametrize("kind,key", [("velocity", "traces_semv"), ("acceleration", "traces_sema")])
def test_oracle_matches_golden_velocity_acceleration(oracle_lib, name, kind, key):
    """Velocity and acceleration traces of the moment-tensor (P-SV) and SH
    fixtures, same metric and tolerance as the displacement traces."""
    import os
    from conftest import GOLDEN
    from oracle import runner
    case, _, _ = golden_case(name)
    traces = np.load(os.path.join(GOLDEN, f"{name}.npz"))[key]
    case.seis_types = [kind]
    r = runner.run(case, "f32", nthreads=8)
    err = reference_metric(r["seis"][:, 0], traces)
    assert np.all(np.isfinite(err))
    assert err.max() < 1e-3, err


def layered_aniso_case(nstep, tilt=True):
    """80 x 60 elastic P-SV mesh (Stacey left/right/bottom): an anisotropic
    lower half (c15, c35 != 0 when ``tilt``) under the isotropic upper half."""
    from oracle import runner
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=nstep)
    rho, vp, vs = 2200.0, 2500.0, 1445.0
    l2m, mu = rho * vp * vp, rho * vs * vs
    mesh = meshgen.structured_mesh(80, 60, 0.0, 4000.0, 0.0, 3000.0,
                                   np.r_[np.zeros(30, np.int32), np.ones(30, np.int32)],
                                   [(1, rho, vp, vs), (1, rho, vp, vs)],
                                   absorbing=("bottom", "right", "left"), free_surface=())
    c = [1.15 * l2m, l2m - 2 * mu, 0.12 * mu, l2m, -0.09 * mu, mu] if tilt else [l2m, l2m - 2 * mu, 0.0, l2m, 0.0, mu]
    mesh.mat_aniso = np.array([c, [np.nan] * 6])
    src = [runner.Source(x=2000.0, z=1300.0, f0=10.0, factor=1e10),
           runner.Source(x=1200.0, z=2500.0, f0=10.0, factor=1e10, angle=30.0)]
    return runner.Case2D(mesh=mesh, sources=src, rec_x=w.rec_x, rec_z=np.r_[np.full(3, 2800.0), np.full(2, 1000.0)],
                         dt=w.dt, nstep=nstep)


def test_oracle_aniso_isotropic_constants_equal_isotropic(oracle_lib):
    """Isotropic constants written as an anisotropic material reproduce the
    isotropic medium (same stress up to FP32 rounding of lambda + 2 mu)."""
    from oracle import runner
    case = layered_aniso_case(500, tilt=False)
    a = runner.run(case, "f32", nthreads=4)["seis"]
    case.mesh.mat_aniso = None
    b = runner.run(case, "f32", nthreads=4)["seis"]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5


def test_oracle_aniso_tilt_changes_wavefield(oracle_lib):
    """c15 / c35 enter the stress: the tilted medium differs from the
    untilted one by far more than rounding."""
    from oracle import runner
    a = runner.run(layered_aniso_case(700, tilt=True), "f32", nthreads=4)["seis"]
    b = runner.run(layered_aniso_case(700, tilt=False), "f32", nthreads=4)["seis"]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) > 1e-2


def test_oracle_fp32_vs_fp64_small(oracle_lib):
    from oracle import runner
    case, _, _ = golden_case("HomogeneousElasticDomainStaceyDirichletBC", nstep=120)
    a = runner.run(case, "f32", nthreads=4)["seis"]
    b = runner.run(case, "f64", nthreads=4)["seis"]
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel < 1e-4


def test_gll_known_answers(oracle_lib):
    L = oracle_lib
    tol = 1e-6
    for x, n, v in [(-1.0, 1, -1.0), (0.0, 1, 0.0), (1.0, 1, 1.0), (-1.0, 2, 1.0), (0.0, 2, -0.5),
                    (1.0, 2, 1.0), (-1.0, 5, -1.0), (0.0, 5, 0.0), (1.0, 5, 1.0)]:
        assert abs(L.oracle_legendre(x, n) - v) < tol
    z = np.zeros(5)
    w = np.zeros(5)
    hp = np.zeros(25)
    dp = C.POINTER(C.c_double)
    L.oracle_gll(z.ctypes.data_as(dp), w.ctypes.data_as(dp), hp.ctypes.data_as(dp))
    assert np.allclose(z, [-1, -np.sqrt(3 / 7), 0, np.sqrt(3 / 7), 1])
    assert np.allclose(w, [0.1, 49 / 90, 32 / 45, 49 / 90, 0.1])
    hp = hp.reshape(5, 5)
    assert np.allclose(hp.sum(axis=1), 0.0, atol=1e-12)    # derivative of a constant
    assert np.allclose(hp @ z, 1.0)                         # derivative of x
    assert np.allclose(hp @ z ** 4, 4 * z ** 3)             # exact up to degree 4


def test_stress_known_answer(oracle_lib):
    kappa, mu = 2.0, 3.0
    du = np.array([1.0, 3.0, 4.0, 2.0])                    # du(0,0), du(0,1), du(1,0), du(1,1)
    out = np.zeros(4)
    dp = C.POINTER(C.c_double)
    oracle_lib.oracle_stress_psv(kappa, mu, du.ctypes.data_as(dp), out.ctypes.data_as(dp))
    lam = kappa + 4.0 / 3.0 * mu - 2 * mu
    assert np.allclose(out, [(lam + 2 * mu) * 1 + lam * 2, mu * 7, mu * 7, (lam + 2 * mu) * 2 + lam * 1])


def golden3d_case(kind="displacement", nstep=None):
    """The 3D fixture (regular 8 x 6 x 6 hexahedra, force source) as an oracle Case3D."""
    import os
    from conftest import GOLDEN
    from oracle import runner3d
    from specfempp_b200 import meshgen
    z = np.load(os.path.join(GOLDEN, "HomogeneousHalfspaceSmallNoABCForceSource.npz"))
    rho, vp, vs = z["material"]
    m = meshgen.homogeneous_hex_mesh(int(z["nex"]), int(z["ney"]), int(z["nez"]), z["extent"], rho, vp, vs)
    fx, fy, fz = z["src_force"]
    src = [runner3d.Source3D(*z["src_xyz"], f0=float(z["src_f0"]), factor=float(z["src_factor"]),
                             comp=(fx, fy, fz, 0.0, 0.0, 0.0), tshift=float(z["src_tshift"]))]
    case = runner3d.Case3D(m, src, z["rec_xyz"], float(z["dt"]), int(nstep or z["nstep"]), [kind])
    return case, z


@pytest.mark.parametrize("kind,key", [("displacement", "traces_semd"), ("velocity", "traces_semv"),
                                      ("acceleration", "traces_sema")])
def test_oracle3d_matches_golden_traces(oracle_lib, kind, key):
    """3D elastic (SPECFEM3D Fortran traces of the reference's dim3 Newmark
    fixture): sum|d|/sum|ref| per station < 1e-3 (observed <= 7e-5)."""
    from oracle import runner3d
    case, z = golden3d_case(kind)
    r = runner3d.run(case, "f32", nthreads=8)
    assert abs(r["t0"] - float(z["trace_t0"])) < 1e-6
    seis = np.transpose(r["seis"][:, 0], (1, 2, 0))     # [nrec, 3, nstep]
    tr = z[key]
    err = np.abs(seis - tr).sum(axis=(1, 2)) / np.abs(tr).sum(axis=(1, 2))
    assert err.max() < 1e-3, err
    assert err.max() < 2e-4


def test_oracle3d_fp32_vs_fp64(oracle_lib):
    from oracle import runner3d
    case, _ = golden3d_case()
    a = runner3d.run(case, "f32", nthreads=4)["seis"]
    b = runner3d.run(case, "f64", nthreads=4)["seis"]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4


COSSERAT_TYPES = {"displacement": ("traces", 2), "velocity": ("traces_semv", 2), "acceleration": ("traces_sema", 2),
                  "pressure": ("traces_semp", 1), "rotation": ("traces_semr", 1),
                  "intrinsic_rotation": ("traces_semir", 1), "curl": ("traces_semc", 1)}


def cosserat_metric(seis, traces, per_station):
    """sum|d| / sum|ref| per station (the reference's metric) or over all
    stations together; seis [nsig, nrec, ncomp], traces [nrec, ncomp, nsig]."""
    if per_station:
        return reference_metric(seis, traces).max()
    n = min(seis.shape[0], traces.shape[2])
    c = np.transpose(seis[:n, :, :traces.shape[1]], (1, 2, 0))
    return float(np.abs(c - traces[:, :, :n]).sum() / np.abs(traces[:, :, :n]).sum())


@pytest.mark.parametrize("name,checks", [
    # the "nu = 0" fixture's database holds an isotropic elastic material:
    # every type of the elastic path at the reference's 1e-3
    ("HomogeneousIsotropicCosseratDomainNu0",
     [("displacement", 1e-3, True), ("velocity", 1e-3, True), ("acceleration", 1e-3, True),
      ("pressure", 1e-3, True)]),
    # nu != 0: the traces come from a finite-difference code (the reference
    # holds them to 1e-1); rotation and curl vanish on the source's symmetry
    # axis, so they are compared over all stations together.  The reference's
    # intrinsic-rotation trace here is its FD rotation minus half the curl, a
    # small difference of nearly equal terms (0.4% of either), and is not used.
    ("HomogeneousIsotropicCosseratDomain",
     [("displacement", 1e-1, True), ("rotation", 1e-1, False), ("curl", 1e-1, False)]),
    # high frequency: the rotation itself is the small term there (its FD trace
    # is 0.1% of the curl's), so curl and intrinsic rotation are compared
    ("HomogeneousIsotropicCosseratDomainHighFrequency",
     [("displacement", 1e-1, True), ("intrinsic_rotation", 1e-1, False), ("curl", 1e-1, False)]),
])
def test_oracle_cosserat_golden(oracle_lib, name, checks):
    """The reference's Cosserat fixtures: the isotropic Cosserat P-SV-T medium
    (displacement + rotation, couple stress) where the database holds one."""
    import os
    from conftest import GOLDEN
    from oracle import runner
    case, _, _ = golden_case(name)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    case.seis_types = [t for t, _, _ in checks]
    r = runner.run(case, "f32", nthreads=8)
    for k, (kind, tol, per_station) in enumerate(checks):
        key, nc = COSSERAT_TYPES[kind]
        err = cosserat_metric(r["seis"][:, k, :, :nc], z[key], per_station)
        assert err < tol, (kind, err)


def cosserat_80x60(nstep, nu_frac=0.1, absorbing=("bottom", "right", "left")):
    """80 x 60 mesh of one isotropic Cosserat material (rho 2200, vp 2500,
    vs 1445 for the displacement part; nu = nu_frac mu; j = rho; lambda_c,
    mu_c, nu_c as fractions of mu like the reference's fixture), Stacey on
    ``absorbing``; a force source, receivers on a line."""
    from oracle import runner
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=nstep)
    rho, vp, vs = 2200.0, 2500.0, 1445.0
    mu = rho * vs * vs
    kappa = rho * vp * vp - 4.0 / 3.0 * mu
    mesh = meshgen.structured_mesh(80, 60, 0.0, 4000.0, 0.0, 3000.0, np.zeros(60, np.int32),
                                   [(1, rho, vp, vs)], absorbing=absorbing, free_surface=())
    mesh.mat_cosserat = np.array([[rho, kappa, mu, nu_frac * mu, rho, 0.0957 * mu, 0.0185 * mu, 0.037 * mu]])
    src = [runner.Source(x=2000.0, z=2000.0, f0=10.0, factor=1e10, angle=20.0)]
    return runner.Case2D(mesh=mesh, sources=src, rec_x=w.rec_x, rec_z=np.full(5, 2600.0), dt=w.dt, nstep=nstep)


def test_oracle_cosserat_nu0_is_elastic(oracle_lib):
    """With nu = 0 the displacement decouples from the rotation: the Cosserat
    medium's displacement equals the isotropic elastic one (FP32 rounding of
    lambda aside), and the rotation stays at rest."""
    from oracle import runner
    case = cosserat_80x60(1200, nu_frac=0.0)      # long enough for the waves to arrive
    case.seis_types = ["displacement", "rotation"]
    a = runner.run(case, "f32", nthreads=8)["seis"]
    case.mesh.mat_cosserat = None
    case.seis_types = ["displacement"]
    b = runner.run(case, "f32", nthreads=8)["seis"]
    assert np.abs(b).max() > 0
    assert np.linalg.norm(a[:, 0] - b[:, 0]) / np.linalg.norm(b[:, 0]) < 1e-5
    assert not np.any(a[:, 1])


def test_oracle_cosserat_nu_couples_rotation(oracle_lib):
    """With nu > 0 the force source excites the rotation, which is bounded
    (the explicit step is stable) and changes the displacement."""
    from oracle import runner
    case = cosserat_80x60(500)
    case.seis_types = ["displacement", "rotation", "curl"]
    a = runner.run(case, "f32", nthreads=8)["seis"]
    assert np.all(np.isfinite(a)) and np.abs(a[:, 1]).max() > 0
    b_case = cosserat_80x60(500, nu_frac=0.0)
    b_case.seis_types = ["displacement"]
    b = runner.run(b_case, "f32", nthreads=8)["seis"]
    assert np.linalg.norm(a[:, 0] - b[:, 0]) / np.linalg.norm(b[:, 0]) > 1e-3


def test_oracle_nonconforming_golden(oracle_lib):
    """The reference's nonconforming fluid-solid fixture (a fine water mesh
    over a coarser elastic one, coupled through 206 nonconforming edge pairs
    each way) against the traces of the conforming run it shares its
    stations and source with, the reference's metric and tolerance 1e-2
    (its config.yaml)."""
    from oracle import runner
    case, traces, t0 = golden_case("AcousticElasticNonconformingCoupledDomain")
    r = runner.run(case, "f32", nthreads=8)
    assert abs(r["t0"] - t0) < 1e-3
    err = reference_metric(r["seis"][:, 0], traces)
    assert np.all(np.isfinite(err))
    assert err.max() < 1e-2, err                          # the reference's tolerance
    assert err.max() < 9e-3                               # observed: 7.8e-3 (elastic side)
    assert np.abs(r["seis"][:, 0, :2]).max() > 0          # elastic receivers reached only by coupling


def test_oracle_nonconforming_coincident_edges_equal_conforming(oracle_lib):
    """Nonconforming records over edges that coincide (equal columns on both
    sides, separate control nodes): the intersection quadrature reduces to
    the GLL points, the transfer functions to the identity, so the run equals
    the conforming twin that shares the interface nodes, to FP64 rounding."""
    from specfempp_b200 import meshgen
    from oracle import runner
    from conftest import workload_case
    w = meshgen.nonconforming_coupled(nx_el=16, nx_ac=16, nz_el=8, nz_ac=6, nstep=700)
    a = runner.run(workload_case(w), "f64", nthreads=8)["seis"][:, 0]
    twin = meshgen.merge_interface_nodes(w.mesh)
    assert len(np.unique(twin.knods)) < len(np.unique(w.mesh.knods))
    w.mesh = twin
    b = runner.run(workload_case(w), "f64", nthreads=8)["seis"][:, 0]
    assert np.abs(b[:, :4]).max() > 0                     # elastic side excited through the interface
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-10


def test_oracle_nonconforming_records_checked(oracle_lib):
    """A nonconforming record without its reverse is refused (the reference's
    symmetry check), as is a record pair whose edges do not overlap."""
    from specfempp_b200 import meshgen
    from oracle import runner
    from conftest import workload_case
    w = meshgen.nonconforming_coupled(nx_el=6, nx_ac=9, nz_el=3, nz_ac=3, nstep=5)
    adj = w.mesh.adjacency
    nc = np.nonzero(adj[:, 2] == 3)[0]
    w.mesh.adjacency = np.delete(adj, nc[0], axis=0)
    with pytest.raises(RuntimeError, match="Non-symmetric"):
        runner.run(workload_case(w), "f32")
    w = meshgen.nonconforming_coupled(nx_el=6, nx_ac=9, nz_el=3, nz_ac=3, nstep=5)
    adj = w.mesh.adjacency.copy()
    e, a = adj[nc[0], 0], adj[nc[0], 1]
    far = a + 8                                            # a water element far from e
    adj[nc[0], 1] = far
    back = np.nonzero((adj[:, 0] == a) & (adj[:, 1] == e))[0][0]
    adj[back, 0] = far
    w.mesh.adjacency = adj
    with pytest.raises(RuntimeError, match="intersection"):
        runner.run(workload_case(w), "f32")


@pytest.mark.parametrize("kind,key", [("displacement", "traces"), ("velocity", "traces_semv"),
                                      ("acceleration", "traces_sema")])
def test_oracle_poroelastic_golden(oracle_lib, kind, key):
    """The reference's poroelastic fixture (fluid-saturated sandstone, four
    components: solid and fluid displacement): solid traces, the reference's
    metric and tolerance 1e-3."""
    import os
    from conftest import GOLDEN
    from oracle import runner
    case, _, t0 = golden_case("PoroelasticCoupledDomainPSV")
    traces = np.load(os.path.join(GOLDEN, "PoroelasticCoupledDomainPSV.npz"))[key]
    case.seis_types = [kind]
    r = runner.run(case, "f32", nthreads=8)
    assert abs(r["t0"] - t0) < 1e-3
    err = reference_metric(r["seis"][:, 0], traces)
    assert np.all(np.isfinite(err))
    assert err.max() < 1e-3, err
    assert err.max() < 1e-4                               # observed: 1.5e-6 / 7.6e-6 / 5.8e-5


def test_oracle_poroelastic_viscous_damping(oracle_lib):
    """A viscous pore fluid (eta_f > 0) damps the wavefield: the run stays
    bounded, differs from the inviscid one, and FP32 tracks FP64."""
    from specfempp_b200 import meshgen
    from oracle import runner
    from conftest import workload_case
    runs = {}
    for eta in (0.0, 1e-3):
        w = meshgen.poroelastic_model(nx=24, nz=24, eta_f=eta, kxz=2e-10, nstep=500, layered=True)
        case = workload_case(w, types=("displacement", "pressure"))
        a = runner.run(case, "f32", nthreads=8)["seis"]
        b = runner.run(case, "f64", nthreads=8)["seis"]
        assert np.all(np.isfinite(a)) and np.abs(b[:, 0]).max() > 0
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4
        runs[eta] = b
    d = np.linalg.norm(runs[1e-3][:, 0] - runs[0.0][:, 0]) / np.linalg.norm(runs[0.0][:, 0])
    assert 1e-3 < d < 0.5, d
