"""Reference-format configuration, stations, sources and trace files (CPU)."""
import os

import numpy as np

from conftest import GOLDEN
from fixture_dir import write_fixture_dir


def test_config_stations_sources_round_trip(tmp_path):
    from specfempp_b200 import io
    cfg_path, z = write_fixture_dir(os.path.join(GOLDEN, "HomogeneousElasticDomainMomentTensor.npz"),
                                    str(tmp_path), types=("displacement", "velocity"))
    cfg = io.read_config(cfg_path)
    assert cfg.nstep == int(z["nstep"]) and abs(cfg.dt - float(z["dt"])) < 1e-15
    assert cfg.elastic_wave == "psv" and cfg.seismogram_types == ["displacement", "velocity"]
    assert os.path.exists(cfg.database) and cfg.output_directory == "traces"
    names, x, zz = io.read_stations(cfg.stations)
    assert len(names) == len(z["rec_x"]) and np.allclose(x, z["rec_x"]) and np.allclose(zz, z["rec_z"])
    (s,) = io.read_sources(cfg.sources)
    assert s.kind == "moment_tensor" and s.mxz == float(z["src"][0][10]) and s.f0 == float(z["src"][0][2])


def test_sh_config_and_channels(tmp_path):
    from specfempp_b200 import io
    cfg_path, _ = write_fixture_dir(os.path.join(GOLDEN, "HomogeneousElasticIsotropicDomainSH.npz"), str(tmp_path))
    assert io.read_config(cfg_path).elastic_wave == "sh"
    assert io.channels("displacement", "sh") == ["BXY"]
    assert io.channels("pressure", "psv") == ["PRE"]


def test_ascii_writer_format(tmp_path):
    from specfempp_b200 import io
    seis = np.arange(3 * 2 * 2 * 2, dtype=np.float32).reshape(3, 2, 2, 2) * 1e-3
    paths = io.write_seismograms_ascii(str(tmp_path), [("AA", "S0001"), ("AA", "S0002")], seis,
                                       ["displacement", "acceleration"], t0=-0.12, dt=1.1e-3, nsb=1)
    assert sorted(os.path.basename(p) for p in paths) == sorted(
        [f"AA.S000{r}.S2.{c}.{e}" for r in (1, 2) for c in ("BXX", "BXZ") for e in ("semd", "sema")])
    a = np.loadtxt(os.path.join(tmp_path, "AA.S0002.S2.BXZ.sema"))
    assert a.shape == (3, 2)
    assert np.allclose(a[:, 0], -0.12 + 1.1e-3 * np.arange(3))
    assert np.allclose(a[:, 1], seis[:, 1, 1, 1], rtol=1e-6)
    line = open(os.path.join(tmp_path, "AA.S0001.S2.BXX.semd")).readline()
    assert line == f"{-0.12:e} {0.0:e}\n"


def test_dataset_ascii_and_npy_layouts(tmp_path):
    """ASCII: <name>.meta ("rank R", "dims d0 d1 ") and one %.10e value per
    line with sub-normal magnitudes written as 0; NPY: Fortran-order header
    with the dataset's dims.  Both read back."""
    from specfempp_b200 import io
    vals = np.array([1.5, -2.25e-3, 1e-42, 3.0e7, 0.0, 7.0], np.float32)
    p = io.write_dataset(str(tmp_path), "A", vals, (3, 2), "ascii")
    assert open(tmp_path / "A.meta").read() == "rank 2\ndims 3 2 \n"
    lines = open(p).read().splitlines()
    assert lines[0] == "1.5000000000e+00" and lines[1] == "-2.2499999031e-03"
    assert lines[2] == "0.0000000000e+00"
    back, dims = io.read_dataset(str(tmp_path), "A")
    assert dims == [3, 2] and np.array_equal(back, np.where(np.abs(vals) < 1.2e-38, 0, vals))
    io.write_dataset(str(tmp_path), "B", vals, (3, 2), "npy")
    arr = np.load(tmp_path / "B.npy")
    assert arr.shape == (3, 2) and np.array_equal(arr, vals.reshape(2, 3).T)   # Fortran order
    back, dims = io.read_dataset(str(tmp_path), "B")
    assert dims == [3, 2] and np.array_equal(back, vals)
    io.write_dataset(str(tmp_path), "C", np.array([True]), (1,), "ascii")
    assert open(tmp_path / "C.txt").read() == "1\n"


def test_kernel_writer_layout_and_formulas(tmp_path):
    """Kernels/<group>/{X, Z, rho, mu, kappa, rhop, alpha, beta}, dims [n][5][5],
    element-tiled order; the derived kernels follow Tromp et al. 2005 Eq. 20."""
    from specfempp_b200 import io, meshgen
    w = meshgen.elastic_psv_80x60(nstep=10)
    m = w.mesh
    x, z, jac = meshgen.gll_geometry(m)
    rng = np.random.default_rng(3)
    shape = (m.nspec, 25)
    rho = np.full(shape, 2200.0)
    kappa, mu = rho * (2500.0 ** 2 - 4 / 3 * 1445.0 ** 2), rho * 1445.0 ** 2
    g = [rng.standard_normal(shape) for _ in range(3)]
    k = io.isotropic_kernels(rho, kappa, mu, *g, jac)
    W = np.outer(meshgen.GLL_WEIGHTS, meshgen.GLL_WEIGHTS).ravel() * jac
    assert np.allclose(k["mu"] * W, mu * g[2])
    assert np.allclose(k["rhop"], k["rho"] + k["kappa"] + k["mu"])
    assert np.allclose(k["alpha"], 2 * (1 + 4 / 3 * mu / kappa) * k["kappa"])
    assert np.allclose(k["beta"], 2 * (k["mu"] - 4 / 3 * mu / kappa * k["kappa"]))
    for lib in ("ascii", "npy"):
        root = io.write_kernels(str(tmp_path / lib), m, k, library=lib)
        grp = os.path.join(root, "elastic_psv_isotropic")
        names = sorted(f.split(".")[0] for f in os.listdir(grp) if not f.endswith(".meta"))
        assert names == sorted(["X", "Z", "rho", "mu", "kappa", "rhop", "alpha", "beta"])
        flat, dims = io.read_dataset(grp, "X")
        assert dims == [m.nspec, 5, 5]
        assert np.allclose(io.from_element_order(flat), x, rtol=1e-6)
        flat, _ = io.read_dataset(grp, "beta")
        assert np.allclose(io.from_element_order(flat), k["beta"].astype(np.float32), rtol=1e-6, atol=0)


class _FakeSim:
    """numbering() and field() of a handle over a mesh, without a GPU."""

    def __init__(self, mesh):
        from specfempp_b200 import meshgen
        x, z, _ = meshgen.gll_geometry(mesh)
        key = np.round(np.stack([x.ravel(), z.ravel()], -1), 6)
        _, ib = np.unique(key, axis=0, return_inverse=True)
        self.ib = ib.reshape(mesh.nspec, 25).astype(np.int32)
        self.n = int(self.ib.max()) + 1
        self.ncomp = 2

    def numbering(self):
        g = np.arange(self.n, dtype=np.int32)
        return self.ib, g, np.full(self.n, -1, np.int32)

    def field(self, medium, which):
        k = {"displacement": 1.0, "velocity": 2.0, "acceleration": 3.0}[which]
        return (k * np.arange(self.n * 2, dtype=np.float32)).reshape(self.n, 2)


def test_wavefield_writer_layout(tmp_path):
    """ForwardWavefield/Coordinates/<medium>/{X, Z, mapping},
    Step<6 digits>/<medium>/{Displacement, Velocity, Acceleration} in
    LayoutLeft order, BoundaryValues/save_boundary_values."""
    from specfempp_b200 import io, meshgen
    m = meshgen.elastic_psv_80x60(nstep=10).mesh
    sim = _FakeSim(m)
    x, _, _ = meshgen.gll_geometry(m)
    for lib in ("ascii", "npy"):
        wr = io.WavefieldWriter(str(tmp_path / lib), sim, m, library=lib)
        wr.initialize()
        wr.write(100)
        wr.finalize()
        coords = os.path.join(wr.root, "Coordinates", "elastic_psv")
        mp, dims = io.read_dataset(coords, "mapping")
        assert dims == [m.nspec, 5, 5]
        mp = mp.reshape(5, 5, m.nspec).transpose(2, 1, 0).reshape(m.nspec, 25).astype(int)   # LayoutLeft
        px, _ = io.read_dataset(coords, "X")
        assert np.allclose(px[mp], x, rtol=1e-6)
        d, dims = io.read_dataset(os.path.join(wr.root, "Step000100", "elastic_psv"), "Velocity")
        assert dims == [sim.n, 2]
        assert np.array_equal(d.reshape(2, sim.n).T, sim.field("elastic", "velocity"))
        b, _ = io.read_dataset(os.path.join(wr.root, "BoundaryValues"), "save_boundary_values")
        assert b.tolist() == [0]


def _with_wavefield_writer(cfg_path, **kw):
    import yaml
    with open(cfg_path) as f:
        cfg = yaml.safe_load(f)
    cfg["parameters"]["simulation-setup"]["simulation-mode"]["forward"]["writer"]["wavefield"] = kw
    with open(cfg_path, "w") as f:
        yaml.safe_dump(cfg, f)


def test_config_wavefield_writer_keys(tmp_path):
    import pytest
    from specfempp_b200 import io
    cfg, _ = write_fixture_dir(os.path.join(GOLDEN, "HomogeneousElasticDomain.npz"), str(tmp_path))
    c = io.read_config(cfg, root=str(tmp_path))
    assert c.wavefield_directory is None
    _with_wavefield_writer(cfg, format="NPY", directory="OUT", **{"time-interval": 50})
    c = io.read_config(cfg, root=str(tmp_path))
    assert (c.wavefield_directory, c.wavefield_format, c.wavefield_interval, c.wavefield_last_step) == \
        ("OUT", "npy", 50, True)
    _with_wavefield_writer(cfg, format="HDF5", directory="OUT")
    with pytest.raises(ValueError, match="HDF5|hdf5"):
        io.read_config(cfg, root=str(tmp_path))
    _with_wavefield_writer(cfg, format="ASCII", directory="OUT", **{"for-adjoint-simulations": True})
    with pytest.raises(ValueError, match="boundary values"):
        io.read_config(cfg, root=str(tmp_path))


def test_time_function_tables_product_vs_oracle():
    """Every time function kind: the library's Python table (the same
    formulas as its C++ set-up) against the oracle's independent restatement,
    both FP32; start times follow each kind's rule."""
    from oracle import runner
    from specfempp_b200 import sfg, stf
    kinds = [("ricker", 10.0, 0.0), ("dirac", 0.0, 0.0), ("gaussian", 8.0, 0.0), ("dgaussian", 12.0, 0.0),
             ("gaussian_hdur", 0.0, 0.02), ("heaviside", 0.0, 0.05), ("heaviside", 0.0, 1e-4)]
    dt, nstep = 5e-4, 600
    for kind, f0, hdur in kinds:
        p = sfg.Source(x=0.0, z=0.0, f0=f0, factor=1e10, tshift=0.01, stf=kind, hdur=hdur)
        o = runner.Source(x=0.0, z=0.0, f0=f0, factor=1e10, tshift=0.01, stf=kind, hdur=hdur)
        a = stf.table([p], dt, nstep)[:, 0]
        b = runner.stf_tables([o], dt, nstep)[:, 0]
        assert np.all(np.isfinite(a)) and np.abs(a).max() > 0, kind
        np.testing.assert_allclose(a, b, rtol=2e-6, atol=2e-6 * np.abs(b).max(), err_msg=kind)
    # start rule of the half-duration kinds: hdur raised to 5 dt, start -2 hdur
    t0, _ = stf.start(sfg.Source(x=0, z=0, f0=0, factor=1, stf="heaviside", hdur=1e-4), dt)
    assert abs(t0 - (-2 * 5 * dt)) < 1e-7


def test_sources_yaml_time_functions(tmp_path):
    import yaml
    from specfempp_b200 import io
    srcs = [{"force": {"x": 1.0, "z": 2.0, "Heaviside": {"hdur": 0.1, "factor": 1e8}}},
            {"force": {"x": 1.0, "z": 2.0, "Gaussian": {"hdur": 0.2, "factor": 1.0}}},
            {"force": {"x": 1.0, "z": 2.0, "Gaussian": {"f0": 3.0, "factor": 1.0}}},
            {"moment-tensor": {"x": 1.0, "z": 2.0, "Mxx": 1.0, "Mzz": 1.0, "Mxz": 0.0,
                               "dGaussian": {"f0": 4.0, "factor": 2.0, "tshift": 0.5}}}]
    p = tmp_path / "sources.yaml"
    p.write_text(yaml.safe_dump({"number-of-sources": len(srcs), "sources": srcs}))
    got = io.read_sources(str(p))
    assert [s.stf for s in got] == ["heaviside", "gaussian_hdur", "gaussian", "dgaussian"]
    assert got[0].hdur == 0.1 and got[2].f0 == 3.0 and got[3].tshift == 0.5 and got[3].kind == "moment_tensor"


def test_given_start_time_table_and_config(tmp_path):
    """A configuration t0 starts the run there with every source's own tshift
    (library table and oracle table agree); config parsing carries it."""
    import yaml
    from oracle import runner
    from specfempp_b200 import io, sfg, stf
    srcs_p = [sfg.Source(x=0, z=0, f0=5.0, factor=1.0, tshift=0.3), sfg.Source(x=0, z=0, f0=8.0, factor=2.0)]
    srcs_o = [runner.Source(x=0, z=0, f0=5.0, factor=1.0, tshift=0.3), runner.Source(x=0, z=0, f0=8.0, factor=2.0)]
    a = stf.table(srcs_p, 1e-3, 800, start_time=-0.5)
    b = runner.stf_tables(srcs_o, 1e-3, 800, start=-0.5)
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6)
    # the Ricker of the second source peaks at t = 0, i.e. step 500
    assert int(np.argmax(a[:, 1])) == 500
    cfg, _ = write_fixture_dir(os.path.join(GOLDEN, "HomogeneousElasticDomain.npz"), str(tmp_path))
    with open(cfg) as f:
        c = yaml.safe_load(f)
    c["parameters"]["simulation-setup"]["solver"]["time-marching"]["time-scheme"]["t0"] = -0.5
    with open(cfg, "w") as f:
        yaml.safe_dump(c, f)
    assert io.read_config(cfg, root=str(tmp_path)).start_time == -0.5
