"""The reference's own adjoint formulation, restated in the oracle
(oracle.runner.adjoint_compat), against the CUDA discrete adjoint.

The reference computes Frechet kernels in a combined run
(core/specfem/solver/time_marching.tpp:133-264): the adjoint field is driven
by adjoint sources at the receivers; the forward field is reconstructed
backwards in time by Newmark with -dt from the saved final state, the Stacey
elements replaying the forward run's contributions; every step adds
kappa_kl = -kappa2D dt div(s+) div(s), mu_kl = -2 mu dt (eps+ : eps - 1/3
div div), rho_kl = -rho dt (s+'' . s) (frechet_derivative.hpp:55-181,
kappa2D = lambda + mu).  These are kernels of relative perturbations,
integrated in time.  For a misfit L = 1/2 sum over steps and receivers of
the squared residual, with the residual as adjoint source, the gradient with
respect to the model at an element GLL point p follows as

    dL/drho_p = rho_kl_p W_p / (rho_p dt),  dL/dmu_p = mu_kl_p W_p / (mu_p dt),
    dL/dkappa_p = kappa_kl_p W_p / (kappa2D_p dt),

W_p = w_x w_z |J| at p, kappa the reference's stored bulk modulus lambda +
2/3 mu (mu at fixed kappa).  The continuous adjoint is O(dt)-accurate: it
matches finite differences of the misfit to 1-2 %, where the CUDA path's
exact discrete adjoint matches them to round-off.

CPU tests (oracle only): the reconstruction reproduces the forward
snapshots to FP64 round-off; the mapped kernels match central finite
differences of the oracle's FP64 misfit within 3e-2; the reference's
two-field gradient (the backward derivatives also receive the adjoint
field's, gradient.hpp:296-317) changes the kernels only by terms quadratic
in the adjoint field, invisible at these amplitudes and visible once the
adjoint sources are scaled up.  GPU test: the CUDA discrete gradient agrees
with the mapped reference kernels along smooth perturbations within 5e-2
(the continuous adjoint's own error, 1-4 % on this model).
"""
import numpy as np
import pytest

NX, NZ, NSTEP = 40, 20, 500


def problem():
    from oracle import runner
    from specfempp_b200 import meshgen
    aw = meshgen.elastic_adjoint_500x250(nstep=NSTEP, nx=NX, nz=NZ, nsrc=1, nrec=10)
    w = aw.workload

    def case_of(rho, kap, mu):
        vp = np.sqrt((kap + 4.0 / 3.0 * mu) / rho)
        vs = np.sqrt(mu / rho)
        return runner.Case2D(mesh=w.mesh, sources=w.sources[:1], rec_x=w.rec_x, rec_z=w.rec_z, dt=w.dt,
                             nstep=NSTEP, point_rho=rho, point_vp=vp, point_vs=vs)

    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    rho_t = f64(aw.true_rho)
    mu_t = rho_t * f64(aw.true_vs) ** 2
    kap_t = rho_t * f64(aw.true_vp) ** 2 - 4.0 / 3.0 * mu_t
    rho0 = f64(w.point_rho)
    mu0 = rho0 * f64(w.point_vs) ** 2
    kap0 = rho0 * f64(w.point_vp) ** 2 - 4.0 / 3.0 * mu0
    obs = runner.run(case_of(rho_t, kap_t, mu_t), "f64", nthreads=8)["seis"][:, 0]
    return aw, case_of, obs, (rho0, kap0, mu0)


def misfit(case_of, obs, m):
    from oracle import runner
    r = runner.run(case_of(*m), "f64", nthreads=8)["seis"][:, 0] - obs
    return 0.5 * float((r * r).sum()), r


def mapped_gradient(k, model, dt):
    rho, kap, mu = model
    W = k["weight"]
    return (k["rho"] * W / (rho * dt), k["kappa"] * W / ((kap + mu / 3.0) * dt), k["mu"] * W / (mu * dt))


def test_reconstruction_equals_forward_snapshots(oracle_lib):
    from oracle import runner
    _, case_of, obs, m0 = problem()
    _, res = misfit(case_of, obs, m0)
    a = runner.adjoint_compat(case_of(*m0), res, reconstruct=True)
    b = runner.adjoint_compat(case_of(*m0), res, reconstruct=False)
    for name in ("rho", "mu", "kappa"):
        assert np.linalg.norm(b[name]) > 0
        assert np.linalg.norm(a[name] - b[name]) <= 1e-10 * np.linalg.norm(b[name]), name


def test_reference_kernels_match_finite_differences(oracle_lib):
    from oracle import runner
    from specfempp_b200 import meshgen
    aw, case_of, obs, m0 = problem()
    _, res = misfit(case_of, obs, m0)
    k = runner.adjoint_compat(case_of(*m0), res)
    g = mapped_gradient(k, m0, aw.workload.dt)
    pert = meshgen.smooth_perturbations(aw.workload.mesh, 25.0 * NX, 25.0 * NZ, 3, 300.0, seed=3)
    h = 1e-4
    for i in range(3):
        d = pert[i] * m0[i]

        def f(hh):
            m = list(m0)
            m[i] = m0[i] + hh * d
            return misfit(case_of, obs, m)[0]
        fd = (f(h) - f(-h)) / (2 * h)
        ad = float((g[i] * d).sum())
        assert abs(ad - fd) <= 3e-2 * abs(fd), (i, ad, fd)


def test_two_field_gradient_quirk(oracle_lib):
    from oracle import runner
    _, case_of, obs, m0 = problem()
    _, res = misfit(case_of, obs, m0)
    plain = runner.adjoint_compat(case_of(*m0), res, quirk=False)
    quirk = runner.adjoint_compat(case_of(*m0), res, quirk=True)
    for name in ("mu", "kappa"):
        assert np.linalg.norm(quirk[name] - plain[name]) <= 1e-9 * np.linalg.norm(plain[name])
    # the added terms are quadratic in the adjoint field: with adjoint sources
    # scaled up to the forward field's size they dominate
    scale = 1e13
    plain = runner.adjoint_compat(case_of(*m0), scale * res, quirk=False)
    quirk = runner.adjoint_compat(case_of(*m0), scale * res, quirk=True)
    for name in ("mu", "kappa"):
        assert np.linalg.norm(quirk[name] - plain[name]) >= 1e-2 * np.linalg.norm(plain[name]), name
    assert np.array_equal(quirk["rho"], plain["rho"])     # rho uses no gradient


@pytest.mark.gpu
def test_cuda_discrete_gradient_against_reference_kernels(sfg_lib, oracle_lib):
    from oracle import runner
    from specfempp_b200 import meshgen, sfg
    aw, case_of, obs, m0 = problem()
    w = aw.workload
    _, res = misfit(case_of, obs, m0)
    k = runner.adjoint_compat(case_of(*m0), res)
    g_ref = mapped_gradient(k, m0, w.dt)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=NSTEP, point_rho=w.point_rho, point_vp=w.point_vp,
                           point_vs=w.point_vs)
    sim.set_sources(w.sources[:1])
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    sim.set_model(*m0)
    sim.forward_checkpointed(NSTEP, 100)
    g_cuda = sim.adjoint_gradient(res.astype(np.float32))
    pert = meshgen.smooth_perturbations(w.mesh, 25.0 * NX, 25.0 * NZ, 6, 300.0, seed=5)
    for i in range(6):
        which = i % 3
        d = pert[i] * m0[which]
        a = float((np.asarray(g_cuda[which], np.float64) * d).sum())
        b = float((g_ref[which] * d).sum())
        print("parameter", ["rho", "kappa", "mu"][which], "cuda", a, "reference kernels", b)
        assert abs(a - b) <= 5e-2 * abs(b), (which, a, b)
    for which in range(3):
        e = np.linalg.norm(np.asarray(g_cuda[which], np.float64) - g_ref[which]) / np.linalg.norm(g_ref[which])
        print("pointwise relative L2", ["rho", "kappa", "mu"][which], e)
        assert e <= 0.25, (which, e)
