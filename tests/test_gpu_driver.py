"""The configuration-file driver end to end on the GPU: a reference-style run
directory rebuilt from a golden fixture, traces written in the reference's
ASCII format and compared with the golden traces (sum|d|/sum|ref| < 1e-3)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fixture_dir import write_fixture_dir

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,comps", [("HomogeneousElasticDomain", ("BXX", "BXZ")),
                                        ("HomogeneousElasticDomainMomentTensor", ("BXX", "BXZ")),
                                        ("HomogeneousElasticIsotropicDomainSH", ("BXY",))])
def test_driver_writes_reference_traces(sfg_lib, tmp_path, name, comps):
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
        assert err / norm < 1e-3, (st, err / norm)
