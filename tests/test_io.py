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
