"""The configuration-file driver end to end on the GPU: a reference-style run
directory rebuilt from a golden fixture, traces written in the reference's
ASCII format and compared with the golden traces (sum|d|/sum|ref| < 1e-3)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fixture_dir import write_fixture_dir

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,comps,tol", [("HomogeneousElasticDomain", ("BXX", "BXZ"), 1e-3),
                                            ("HomogeneousElasticDomainMomentTensor", ("BXX", "BXZ"), 1e-3),
                                            ("HomogeneousElasticDomainMomentTensorHeaviside", ("BXX", "BXZ"), 1e-3),
                                            ("HomogeneousElasticIsotropicDomainSH", ("BXY",), 1e-3),
                                            ("PoroelasticCoupledDomainPSV", ("BXX", "BXZ"), 1e-3),
                                            ("AcousticElasticNonconformingCoupledDomain", ("BXX", "BXZ"), 1e-2)])
def test_driver_writes_reference_traces(sfg_lib, tmp_path, name, comps, tol):
    from specfempp_b200 import specfem2d
    cfg, z = write_fixture_dir(os.path.join(GOLDEN, f"{name}.npz"), str(tmp_path))
    out = specfem2d.run_config(cfg, root=str(tmp_path))
    assert out["files"] == len(z["stations"]) * len(comps)
    for r, st in enumerate(z["stations"]):
        err = norm = 0.0
        for c, ch in enumerate(comps):
            t, v = np.loadtxt(os.path.join(out["output_directory"], f"{st}.S2.{ch}.semd")).T
            ref = z["traces"][r, c]
            n = min(len(v), len(ref))
            err += np.abs(v[:n] - ref[:n]).sum()
            norm += np.abs(ref[:n]).sum()
            assert abs(t[0] - float(z["trace_t0"])) < 1e-6
        assert err / norm < tol, (st, err / norm)


@pytest.mark.parametrize("library", ["ascii", "npy"])
def test_driver_wavefield_snapshots(sfg_lib, tmp_path, library):
    """A configuration with a wavefield writer: snapshots after every
    time-interval steps and at the last step, in the ForwardWavefield layout;
    the last snapshot is the field of a plain run of the same model, bit for
    bit, at every element point (ASCII, like the reference's writer, writes
    magnitudes below the smallest normal float as 0)."""
    import yaml
    from specfempp_b200 import io, specfem2d, sfg
    from test_io import _with_wavefield_writer
    cfg, z = write_fixture_dir(os.path.join(GOLDEN, "HomogeneousElasticDomain.npz"), str(tmp_path))
    nstep = 300
    with open(cfg) as f:
        c = yaml.safe_load(f)
    c["parameters"]["simulation-setup"]["solver"]["time-marching"]["time-scheme"]["nstep"] = nstep
    with open(cfg, "w") as f:
        yaml.safe_dump(c, f)
    os.makedirs(tmp_path / "OUT")
    _with_wavefield_writer(cfg, format=library.upper(), directory="OUT", **{"time-interval": 120})
    out = specfem2d.run_config(cfg, root=str(tmp_path))
    assert out["wavefield_steps"] == [120, 240, 300]
    root = tmp_path / "OUT" / "ForwardWavefield"
    assert sorted(os.listdir(root)) == ["BoundaryValues", "Coordinates", "Step000120", "Step000240", "Step000300"]
    coords = str(root / "Coordinates" / "elastic_psv")
    mp, dims = io.read_dataset(coords, "mapping")
    n = int(dims[0])
    mp = mp.reshape(5, 5, n).transpose(2, 1, 0).reshape(n, 25).astype(int)
    d, dims = io.read_dataset(str(root / "Step000300" / "elastic_psv"), "Displacement")
    d = d.reshape(2, dims[0]).T
    # plain run of the same configuration
    cf = io.read_config(cfg, root=str(tmp_path))
    stations, rx, rz = io.read_stations(cf.stations)
    sim = sfg.Simulation2D(database=cf.database, dt=cf.dt, nstep=nstep)
    sim.set_sources(io.read_sources(cf.sources))
    sim.set_receivers(rx, rz)
    sim.initialize()
    sim.run(nstep)
    ib, g2e, _ = sim.numbering()
    u = sim.field("elastic")
    assert np.abs(u).max() > 0
    want = u[g2e[ib]]
    if library == "ascii":
        want = np.where(np.abs(want) < np.finfo(np.float32).tiny, 0.0, want).astype(np.float32)
    assert np.array_equal(d[mp], want)
    x, _, _, _ = sim.geometry()
    px, _ = io.read_dataset(coords, "X")
    assert np.allclose(px[mp], x, rtol=1e-6)
