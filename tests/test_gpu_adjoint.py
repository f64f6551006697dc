"""Discrete-adjoint model gradients (2D elastic P-SV, SH, acoustic and coupled
acoustic-elastic) against finite differences.

The gradient of L = sum(w * seis) for a seeded weight array w is checked,
along smooth Gaussian perturbations of rho, kappa and mu placed between the
source and the receivers, and on the absorbing edge (where the Stacey
impedances depend on the model), against central differences of two forward runs:
relative error <= 1e-2 (the FP32 forward limits the difference quotient to
about 1e-3 at a 1% perturbation).  Gradients from different checkpoint
intervals agree to 1e-5 (only the order of the FP32 time sum differs); the
memory budget of the recorded segments changes no bit.  Coupled
acoustic-elastic models are checked against FP64-oracle differences.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSTEP = 600


def setup(w):
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=NSTEP)
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    return sim


def base_model(mesh):
    nspec = mesh.nspec
    m = mesh.kmato
    rho = np.repeat(mesh.mat_rho[m][:, None], 25, 1)
    vp = np.repeat(mesh.mat_vp[m][:, None], 25, 1)
    vs = np.repeat(mesh.mat_vs[m][:, None], 25, 1)
    mu = rho * vs ** 2
    kappa = rho * vp ** 2 - 4.0 / 3.0 * mu
    return [np.ascontiguousarray(a.reshape(nspec, 25), np.float64) for a in (rho, kappa, mu)]


def bump(mesh, x0, z0, sigma):
    from specfempp_b200 import meshgen
    z, x = meshgen.gll_coordinates(mesh)
    return np.exp(-((x - x0) ** 2 + (z - z0) ** 2) / (2 * sigma ** 2))


@pytest.fixture(scope="module")
def problem(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_psv_80x60(nstep=NSTEP)
    sim = setup(w)
    model = base_model(w.mesh)
    nrec = len(w.rec_x)
    weights = np.random.default_rng(11).standard_normal((NSTEP, nrec, 2)).astype(np.float32)
    return w, sim, model, weights


def misfit(sim, model, weights):
    sim.set_model(*[m.astype(np.float32) for m in model])
    seis = sim.forward_checkpointed(NSTEP, 50).astype(np.float64)
    return float((seis * weights).sum())


def gradient(sim, model, weights, interval):
    sim.set_model(*[m.astype(np.float32) for m in model])
    sim.forward_checkpointed(NSTEP, interval)
    return sim.adjoint_gradient(weights)


@pytest.mark.parametrize("which", [0, 1, 2], ids=["rho", "kappa", "mu"])
def test_adjoint_matches_finite_differences(problem, which):
    w, sim, model, weights = problem
    g = gradient(sim, model, weights, 50)[which].astype(np.float64)
    d = bump(w.mesh, 2000.0, 2650.0, 250.0) * model[which]
    eps = 1e-2
    plus = [m.copy() for m in model]
    minus = [m.copy() for m in model]
    plus[which] += eps * d
    minus[which] -= eps * d
    fd = (misfit(sim, plus, weights) - misfit(sim, minus, weights)) / (2 * eps)
    ad = float((g * d).sum())
    assert abs(fd) > 0
    assert abs(ad - fd) <= 1e-2 * abs(fd), (ad, fd, abs(ad - fd) / abs(fd))


def test_checkpoint_interval_invariance(problem):
    w, sim, model, weights = problem
    a = gradient(sim, model, weights, 1)
    b = gradient(sim, model, weights, 37)
    c = gradient(sim, model, weights, NSTEP)
    for x, y, z in zip(a, b, c):
        n = np.linalg.norm(x)
        assert n > 0
        assert np.linalg.norm(x - y) <= 1e-5 * n
        assert np.linalg.norm(x - z) <= 1e-5 * n


def test_segment_budget_gives_the_same_gradient(problem):
    """Two segment buffers (the forward run keeps its last two segments, the
    reverse sweep recomputes the others) and the default budget (every
    segment kept from the forward run) give the same bits; so does a second
    gradient without a new forward run (everything recomputed)."""
    w, sim, model, weights = problem
    nseg = -(-NSTEP // 37)
    sim.set_adjoint_budget(1)
    a = gradient(sim, model, weights, 37)
    assert sim.adjoint_buffers() == 2
    sim.set_adjoint_budget(0)
    b = gradient(sim, model, weights, 37)
    assert sim.adjoint_buffers() == nseg
    c = sim.adjoint_gradient(weights)
    for x, y, z in zip(a, b, c):
        assert np.abs(x).max() > 0
        assert np.array_equal(x, y)
        assert np.array_equal(x, z)


def test_row_form_reverse_kernel_gives_the_same_gradient(sfg_lib):
    """kernel_variant 6 (row-form element kernels, forward and reverse) and 3
    (point form): the same gradient bits."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=NSTEP)
    model = base_model(w.mesh)
    weights = np.random.default_rng(17).standard_normal((NSTEP, len(w.rec_x), 2)).astype(np.float32)
    out = []
    for v in (3, 6):
        sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=NSTEP, kernel_variant=v)
        sim.set_sources(w.sources)
        sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
        sim.initialize()
        assert sim.info().kernel_variant == v
        out.append(gradient(sim, model, weights, 50))
        sim.close()
    for x, y in zip(*out):
        assert np.abs(x).max() > 0
        assert np.array_equal(x, y)


def test_autograd_function(problem):
    import torch
    from specfempp_b200 import adjoint
    w, sim, model, weights = problem
    t = [torch.tensor(m, dtype=torch.float32, requires_grad=True) for m in model]
    seis = adjoint.seismograms(sim, *t, nsteps=NSTEP, interval=50)
    loss = (seis * torch.from_numpy(weights)).sum()
    loss.backward()
    g = gradient(sim, model, weights, 50)
    for ti, gi in zip(t, g):
        assert np.array_equal(ti.grad.numpy(), gi)


def test_adjoint_rejects_unsupported(sfg_lib):
    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=50)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=50)
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_x, w.rec_z, types=("velocity",))
    sim.initialize()
    with pytest.raises(sfg.SfgError):
        sim.forward_checkpointed(50, 10)
    sim2 = setup(meshgen.elastic_psv_80x60(nstep=NSTEP))
    with pytest.raises(sfg.SfgError):
        sim2.adjoint_gradient(np.zeros((NSTEP, 5, 2), np.float32))


def fd4(f, h):
    """Fourth-order central difference of f at 0."""
    return (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)


def small_inversion():
    from specfempp_b200 import adjoint, meshgen, sfg
    aw = meshgen.elastic_adjoint_500x250(nstep=800, nx=100, nz=50, nsrc=2, nrec=20, seed=1)
    w = aw.workload
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep, point_rho=w.point_rho, point_vp=w.point_vp,
                           point_vs=w.point_vs)
    sim.set_sources([w.sources[0]])
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    kt, mt = adjoint.moduli(aw.true_rho.astype(np.float64), aw.true_vp.astype(np.float64),
                            aw.true_vs.astype(np.float64))
    obs = adjoint.observed_data(sim, w.sources, aw.true_rho, kt, mt, w.nstep)
    rho0 = w.point_rho.astype(np.float64)
    k0, m0 = adjoint.moduli(rho0, w.point_vp.astype(np.float64), w.point_vs.astype(np.float64))
    return aw, sim, obs, [rho0, k0, m0]


def test_l2_misfit_gradient_matches_fd4(sfg_lib):
    """Summed two-source L2 waveform misfit: adjoint directional derivatives
    against fourth-order central differences (step 0.5% of the model along the
    perturbation) along seeded smooth perturbations of each parameter that
    reach the absorbing edges, relative error <= 1e-3."""
    from specfempp_b200 import adjoint, meshgen
    aw, sim, obs, model = small_inversion()
    w = aw.workload
    L, grads = adjoint.l2_misfit_gradient(sim, w.sources, *model, obs, w.nstep, 100)
    assert L > 0
    pert = meshgen.smooth_perturbations(w.mesh, 2500.0, 1250.0, 3, 500.0, seed=5)
    for which in range(3):
        d = pert[which] * model[which]

        def f(h):
            m = [x.copy() for x in model]
            m[which] = m[which] + h * d
            return adjoint.l2_misfit(sim, w.sources, *m, obs, w.nstep)
        fd = fd4(f, 0.005)
        ad = float((grads[which] * d).sum())
        assert abs(ad - fd) <= 1e-3 * abs(fd), (which, ad, fd, abs(ad - fd) / abs(fd))


def test_sources_replaced_after_initialize(sfg_lib):
    """Replacing the source of an initialised handle gives the same bits as a
    handle created with that source."""
    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=300)
    other = meshgen.RickerSource(1200.0, 1500.0, 12.0, 1e10)
    a = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=300)
    a.set_sources(w.sources)
    a.set_receivers(w.rec_x, w.rec_z)
    a.initialize()
    a.run(300)
    a.set_sources([other])
    a.reset()
    a.run(300)
    b = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=300)
    b.set_sources([other])
    b.set_receivers(w.rec_x, w.rec_z)
    b.initialize()
    b.run(300)
    assert np.array_equal(a.seismograms(), b.seismograms())
    with pytest.raises(sfg.SfgError):
        a.set_sources([other, other])


@pytest.mark.parametrize("interval", [50, 37, NSTEP])
def test_checkpointed_forward_equals_plain_run(problem, interval):
    """The checkpointed forward (its last segment recorded on the way) gives
    the plain run's seismograms bit for bit."""
    w, sim, model, weights = problem
    sim.set_model(*[m.astype(np.float32) for m in model])
    sim.reset()
    sim.run(NSTEP)
    plain = sim.seismograms()[0, :, 0].copy()
    ck = sim.forward_checkpointed(NSTEP, interval)
    assert np.array_equal(plain, ck)


def test_kernel_files_from_the_gradient(problem, tmp_path):
    """Relative kernels from the gradient, written in the reference's Kernels
    layout: sum of W K_m dln(m) equals the gradient's directional derivative
    along m dln(m); the NPY files read back to the kernels."""
    from specfempp_b200 import io, meshgen
    w, sim, model, weights = problem
    g = [a.astype(np.float64) for a in gradient(sim, model, weights, 50)]
    x, z, jac, med = sim.geometry()
    k = io.isotropic_kernels(*model, *g, jac)
    W = np.outer(meshgen.GLL_WEIGHTS, meshgen.GLL_WEIGHTS).ravel() * jac
    d = bump(w.mesh, 2000.0, 2650.0, 250.0)
    for name, which in (("rho", 0), ("kappa", 1), ("mu", 2)):
        lhs = float((W * k[name] * d).sum())
        rhs = float((g[which] * model[which] * d).sum())
        assert abs(lhs - rhs) <= 1e-9 * abs(rhs), name
    root = io.write_kernels(str(tmp_path), sim, k, library="npy")
    for name in ("rho", "kappa", "mu", "rhop", "alpha", "beta"):
        flat, dims = io.read_dataset(f"{root}/elastic_psv_isotropic", name)
        assert dims == [w.mesh.nspec, 5, 5]
        assert np.array_equal(io.from_element_order(flat), k[name].astype(np.float32)), name


@pytest.fixture(scope="module")
def problem_sh(sfg_lib):
    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=NSTEP)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=NSTEP, elastic_wave="sh")
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    model = base_model(w.mesh)
    weights = np.random.default_rng(12).standard_normal((NSTEP, len(w.rec_x), 2)).astype(np.float32)
    return w, sim, model, weights


EDGE_NSTEP = 1400


def edge_problem(wave):
    """80 x 60 elastic mesh, Stacey left/right/bottom: a source 700 m from the
    absorbing left edge and receivers between the two, run long enough
    (1400 steps, 0.7 s) for the waves to reach the edge and come back."""
    from dataclasses import replace
    from specfempp_b200 import meshgen, sfg
    w = meshgen.elastic_psv_80x60(nstep=EDGE_NSTEP)
    srcs = [replace(w.sources[0], x=700.0, z=1500.0)]
    rx = np.array([300.0, 500.0, 900.0, 1300.0, 1700.0])
    rz = np.array([2000.0, 1000.0, 2200.0, 800.0, 1500.0])
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=EDGE_NSTEP, elastic_wave=wave)
    sim.set_sources(srcs)
    sim.set_receivers(rx, rz, types=("displacement",))
    sim.initialize()
    weights = np.random.default_rng(13).standard_normal((EDGE_NSTEP, len(rx), 2)).astype(np.float32)
    return w, sim, base_model(w.mesh), weights


def _fd_check(w, sim, model, weights, which, x0, z0, sigma, nstep=NSTEP, order4=False):
    def mis(m):
        sim.set_model(*[a.astype(np.float32) for a in m])
        seis = sim.forward_checkpointed(nstep, 50).astype(np.float64)
        return float((seis * weights).sum())
    sim.set_model(*[m.astype(np.float32) for m in model])
    sim.forward_checkpointed(nstep, 50)
    g = sim.adjoint_gradient(weights)[which].astype(np.float64)
    d = bump(w.mesh, x0, z0, sigma) * model[which]
    eps = 1e-2

    def f(h):
        m = [a.copy() for a in model]
        m[which] += h * d
        return mis(m)
    fd = fd4(f, eps) if order4 else (f(eps) - f(-eps)) / (2 * eps)
    ad = float((g * d).sum())
    return ad, fd


@pytest.mark.parametrize("which", [0, 2], ids=["rho", "mu"])
def test_sh_adjoint_matches_finite_differences(problem_sh, which):
    """SH (u_y, sigma = mu grad u_y): the rho and mu gradients along a smooth
    bump between source and receivers against central differences (relative
    1e-2 as for P-SV); the kappa gradient is zero."""
    w, sim, model, weights = problem_sh
    ad, fd = _fd_check(w, sim, model, weights, which, 2000.0, 2650.0, 250.0)
    assert abs(fd) > 0
    assert abs(ad - fd) <= 1e-2 * abs(fd), (ad, fd, abs(ad - fd) / abs(fd))
    gk = gradient(sim, model, weights, 50)[1]
    assert not np.any(gk)


@pytest.mark.parametrize("wave,which", [("psv", 0), ("psv", 1), ("psv", 2), ("sh", 0), ("sh", 2)],
                         ids=["psv-rho", "psv-kappa", "psv-mu", "sh-rho", "sh-mu"])
def test_adjoint_fd_on_absorbing_edge(sfg_lib, wave, which):
    """A bump on the absorbing left edge, where the Stacey impedances (rho vp
    and rho vs in P-SV, rho vs in SH) depend on the model, against central
    differences (relative 1e-2)."""
    w, sim, model, weights = edge_problem(wave)
    ad, fd = _fd_check(w, sim, model, weights, which, 100.0, 1500.0, 250.0, nstep=EDGE_NSTEP)
    big, _ = _fd_check(w, sim, model, weights, which, 1100.0, 1500.0, 250.0, nstep=EDGE_NSTEP)
    assert abs(fd) > 1e-3 * abs(big), (fd, big)          # the edge matters to the misfit
    assert abs(ad - fd) <= 1e-2 * abs(fd), (ad, fd, abs(ad - fd) / abs(fd))


def test_sh_checkpoint_interval_invariance(problem_sh):
    w, sim, model, weights = problem_sh
    a = gradient(sim, model, weights, 1)
    b = gradient(sim, model, weights, 37)
    for x, y in ((a[0], b[0]), (a[2], b[2])):
        n = np.linalg.norm(x)
        assert n > 0
        assert np.linalg.norm(x - y) <= 1e-5 * n


def acoustic_problem(src_x=2000.0, src_z=1500.0, nstep=NSTEP, rec_z=None):
    """80 x 60 acoustic mesh (vp 1500, rho 1020), free surface on top, Stacey
    on the other sides, a pressure (force) source and pressure receivers."""
    from dataclasses import replace
    from specfempp_b200 import meshgen, sfg
    mesh = meshgen.structured_mesh(80, 60, 0.0, 4000.0, 0.0, 3000.0, np.zeros(60, np.int32),
                                   [(meshgen.ACOUSTIC, 1020.0, 1500.0, 0.0)],
                                   absorbing=("bottom", "right", "left"), free_surface=("top",))
    w = replace(meshgen.elastic_psv_80x60(nstep=nstep), mesh=mesh)
    srcs = [replace(w.sources[0], x=src_x, z=src_z)]
    rx = np.array([300.0, 900.0, 1700.0, 2500.0, 3300.0])
    rz = np.array([2700.0, 2000.0, 2900.0, 1200.0, 2500.0]) if rec_z is None else np.asarray(rec_z)
    sim = sfg.Simulation2D(mesh, dt=w.dt, nstep=nstep)
    sim.set_sources(srcs)
    sim.set_receivers(rx, rz, types=("pressure",))
    sim.initialize()
    weights = np.random.default_rng(14).standard_normal((nstep, len(rx), 2)).astype(np.float32)
    return w, sim, base_model(mesh), weights


# (source, bump, reference bump near the source, steps, receiver depths)
ACOUSTIC_CASES = {
    "interior": ((2000.0, 1500.0), (2000.0, 1800.0), (2000.0, 1500.0), NSTEP, None),
    "free_surface": ((2000.0, 2750.0), (2000.0, 2950.0), (2000.0, 2700.0), NSTEP,
                     [2850.0, 2700.0, 2900.0, 2600.0, 2800.0]),
    "absorbing_edge": ((700.0, 1500.0), (100.0, 1500.0), (1100.0, 1500.0), EDGE_NSTEP, None),
}


@pytest.mark.parametrize("which", [0, 1], ids=["rho", "kappa"])
@pytest.mark.parametrize("where", ["interior", "free_surface"])
def test_acoustic_adjoint_matches_finite_differences(sfg_lib, which, where):
    """Acoustic medium with pressure seismograms: the rho and kappa gradients
    along smooth bumps in the interior and just under the free surface
    (Dirichlet points masked; the bump reaches the source, whose array l /
    kappa depends on kappa), against FP32 central differences (relative
    1e-2); each bump's effect on the misfit is checked to be well above the
    difference quotient's noise.  On the absorbing edge the FP32 quotient
    itself is off by about 1% (the edge moves the misfit little), so that
    case is checked against the FP64 oracle below."""
    (sx, sz), (x0, z0), (bx, bz), nstep, rz = ACOUSTIC_CASES[where]
    w, sim, model, weights = acoustic_problem(sx, sz, nstep, rz)
    # fourth-order differences next to the source, where the response to a 1%
    # change is curved enough to move a second-order quotient by about 2%
    ad, fd = _fd_check(w, sim, model, weights, which, x0, z0, 250.0, nstep=nstep,
                       order4=where == "free_surface")
    big, _ = _fd_check(w, sim, model, weights, which, bx, bz, 250.0, nstep=nstep)
    assert abs(fd) > 1e-3 * abs(big), (fd, big)
    assert abs(ad - fd) <= 1e-2 * abs(fd), (ad, fd, abs(ad - fd) / abs(fd))


@pytest.mark.parametrize("which", [0, 1], ids=["rho", "kappa"])
@pytest.mark.parametrize("where", ["free_surface", "absorbing_edge"])
def test_acoustic_adjoint_vs_fp64_oracle_differences(sfg_lib, oracle_lib, which, where):
    """Directional derivatives under the free surface and on the absorbing
    edge against central differences of the FP64 CPU oracle at a 0.1% step
    (curvature and FP32 noise out of the way): relative 1e-3 (observed below
    1e-4)."""
    from oracle import runner
    (sx, sz), (x0, z0), _, nstep, rz = ACOUSTIC_CASES[where]
    w, sim, model, weights = acoustic_problem(sx, sz, nstep, rz)
    sim.set_model(*[m.astype(np.float32) for m in model])
    sim.forward_checkpointed(nstep, 50)
    g = sim.adjoint_gradient(weights)[which].astype(np.float64)
    d = bump(w.mesh, x0, z0, 250.0) * model[which]
    src = [runner.Source(x=sx, z=sz, f0=w.sources[0].f0, factor=w.sources[0].factor)]
    rx = np.array([300.0, 900.0, 1700.0, 2500.0, 3300.0])
    rzz = np.array([2700.0, 2000.0, 2900.0, 1200.0, 2500.0]) if rz is None else np.asarray(rz)

    def L(h):
        rho, kap = model[0].copy(), model[1].copy()
        (rho if which == 0 else kap)[...] += h * d
        vp = np.sqrt(kap / rho)
        case = runner.Case2D(mesh=w.mesh, sources=src, rec_x=rx, rec_z=rzz, dt=w.dt, nstep=nstep,
                             seis_types=["pressure"], point_rho=rho, point_vp=vp, point_vs=np.zeros_like(vp))
        s = runner.run(case, "f64", nthreads=8)["seis"][:, 0]
        return float((s[:nstep] * weights).sum())
    fd = (L(1e-3) - L(-1e-3)) / 2e-3
    ad = float((g * d).sum())
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd, abs(ad - fd) / abs(fd))


def test_acoustic_mu_enters_as_bulk_modulus(sfg_lib):
    """The acoustic medium uses kappa + 4/3 mu as its bulk modulus, so the
    gradient with respect to mu is 4/3 of the one with respect to kappa."""
    w, sim, model, weights = acoustic_problem()
    g = gradient(sim, model, weights, 50)
    assert np.abs(g[1]).max() > 0
    scale = float(np.abs(g[1]).max())
    assert np.allclose(g[2], (4.0 / 3.0) * g[1].astype(np.float64), rtol=1e-6, atol=1e-6 * scale)


def test_acoustic_checkpoint_interval_invariance(sfg_lib):
    w, sim, model, weights = acoustic_problem()
    a = gradient(sim, model, weights, 1)
    b = gradient(sim, model, weights, 37)
    for x, y in ((a[0], b[0]), (a[1], b[1])):
        n = np.linalg.norm(x)
        assert n > 0
        assert np.linalg.norm(x - y) <= 1e-5 * n


# --------------------------------------------------------------------------
# Coupled acoustic-elastic models (conforming interface): the discrete
# adjoint of the coupled step (transposed coupling terms in both directions).

COUPLED_NSTEP = 700


def coupled_problem(kind, nstep=COUPLED_NSTEP):
    """60 x 50 model over 3000 x 2500 m: 30 elastic rows (rho 2300, vp 3000,
    vs 1730) under 20 water rows (rho 1020, vp 1500), seafloor at z = 1500 m,
    free surface on top, Stacey on the other sides; a pressure source in the
    water 250 m above the seafloor and a force source in the solid; receivers
    50 m under the seafloor (displacement) or 100 m above it (pressure)."""
    from specfempp_b200 import meshgen, sfg
    rows = np.zeros(50, np.int32)
    rows[30:] = 1
    mesh = meshgen.structured_mesh(60, 50, 0.0, 3000.0, 0.0, 2500.0, rows,
                                   [(meshgen.ELASTIC, 2300.0, 3000.0, 1730.0), (meshgen.ACOUSTIC, 1020.0, 1500.0, 0.0)],
                                   absorbing=("bottom", "right", "left"), free_surface=("top",))
    srcs = [meshgen.RickerSource(1500.0, 1750.0, 12.0, 1e10), meshgen.RickerSource(900.0, 1100.0, 12.0, 1e9,
                                                                                  angle=30.0)]
    rx = np.array([600.0, 1100.0, 1900.0, 2400.0])
    rz = np.full(4, 1450.0 if kind == "displacement" else 1600.0)
    sim = sfg.Simulation2D(mesh, dt=4e-4, nstep=nstep)
    sim.set_sources(srcs)
    sim.set_receivers(rx, rz, types=(kind,))
    sim.initialize()
    weights = np.random.default_rng(17).standard_normal((nstep, len(rx), 2)).astype(np.float32)
    return mesh, sim, base_model(mesh), weights


# (parameter, bump centre, radius): in the water, in the solid, across the seafloor
COUPLED_BUMPS = {"water_rho": (0, (1300.0, 1650.0), 120.0), "water_kappa": (1, (1300.0, 1650.0), 120.0),
                 "solid_rho": (0, (1700.0, 1250.0), 150.0), "solid_kappa": (1, (1700.0, 1250.0), 150.0),
                 "solid_mu": (2, (1700.0, 1250.0), 150.0), "seafloor_rho": (0, (1200.0, 1500.0), 150.0)}


def coupled_oracle_misfit(mesh, kind, model, weights, which, d, h):
    """The misfit of the FP64 CPU oracle for the model moved by h * d."""
    from oracle import runner
    m = [x.copy() for x in model]
    m[which] = m[which] + h * d
    rho, kap, mu = m
    vp = np.sqrt((kap + 4.0 / 3.0 * mu) / rho)
    vs = np.sqrt(mu / rho)
    src = [runner.Source(x=1500.0, z=1750.0, f0=12.0, factor=1e10),
           runner.Source(x=900.0, z=1100.0, f0=12.0, factor=1e9, angle=30.0)]
    rx = np.array([600.0, 1100.0, 1900.0, 2400.0])
    rz = np.full(4, 1450.0 if kind == "displacement" else 1600.0)
    case = runner.Case2D(mesh=mesh, sources=src, rec_x=rx, rec_z=rz, dt=4e-4, nstep=COUPLED_NSTEP,
                         seis_types=[kind], point_rho=rho, point_vp=vp, point_vs=vs)
    s = runner.run(case, "f64", nthreads=8)["seis"][:, 0]
    return float((s[:COUPLED_NSTEP] * weights).sum())


@pytest.mark.parametrize("kind", ["displacement", "pressure"])
@pytest.mark.parametrize("case", list(COUPLED_BUMPS))
def test_coupled_adjoint_matches_finite_differences(sfg_lib, oracle_lib, kind, case):
    """Coupled model, displacement seismograms at solid receivers or pressure
    seismograms at water receivers: the gradient along smooth bumps in the
    water, in the solid and across the seafloor against central differences
    of the FP64 CPU oracle at a 0.1% step: relative 1e-3 (observed about
    1e-6).  FP32 differences of the product's own forward runs are too noisy
    here: the water receivers' misfit is about 1e4 times its sensitivity to
    the solid bumps."""
    mesh, sim, model, weights = coupled_problem(kind)
    which, (x0, z0), r = COUPLED_BUMPS[case]
    sim.set_model(*[m.astype(np.float32) for m in model])
    sim.forward_checkpointed(COUPLED_NSTEP, 50)
    g = sim.adjoint_gradient(weights)[which].astype(np.float64)
    d = bump(mesh, x0, z0, r) * model[which]
    fd = (coupled_oracle_misfit(mesh, kind, model, weights, which, d, 1e-3) -
          coupled_oracle_misfit(mesh, kind, model, weights, which, d, -1e-3)) / 2e-3
    ad = float((g * d).sum())
    assert abs(fd) > 0
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd, abs(ad - fd) / abs(fd))


@pytest.mark.parametrize("kind", ["displacement", "pressure"])
def test_coupled_checkpoint_interval_and_budget(sfg_lib, kind):
    """Coupled sweep: gradients from checkpoint intervals 1, 37 and the whole
    run agree to 1e-5; two segment buffers and the default budget give the
    same bits."""
    mesh, sim, model, weights = coupled_problem(kind, nstep=300)
    sim.set_model(*[m.astype(np.float32) for m in model])

    def grad(interval):
        sim.forward_checkpointed(300, interval)
        return sim.adjoint_gradient(weights)
    a, b, c = grad(1), grad(37), grad(300)
    for x, y, z in zip(a, b, c):
        n = np.linalg.norm(x)
        assert n > 0
        assert np.linalg.norm(x - y) <= 1e-5 * n
        assert np.linalg.norm(x - z) <= 1e-5 * n
    sim.set_adjoint_budget(1)
    p = grad(37)
    assert sim.adjoint_buffers() == 2
    sim.set_adjoint_budget(0)
    q = grad(37)
    for x, y in zip(p, q):
        assert np.array_equal(x, y)


def test_coupled_adjoint_refusals(sfg_lib):
    """Displacement seismograms at water receivers (or pressure at solid
    ones) have no adjoint here: SFG_ERR_UNSUPPORTED, nothing run."""
    from specfempp_b200 import sfg
    mesh, sim, model, weights = coupled_problem("displacement", nstep=50)
    sim2 = sfg.Simulation2D(mesh, dt=4e-4, nstep=50)
    sim2.set_sources([sfg.Source(x=1500.0, z=1750.0, f0=12.0, factor=1e10)])
    sim2.set_receivers(np.array([600.0]), np.array([1600.0]), types=("displacement",))
    sim2.initialize()
    with pytest.raises(sfg.SfgError, match="coupled adjoint"):
        sim2.forward_checkpointed(50, 10)
