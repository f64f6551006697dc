"""Full-size configurations through size-independent properties (the oracle
is too slow at these sizes):

* linearity: doubling every source factor doubles every seismogram sample to
  FP32 precision.  A power-of-two scale commutes with every FP32 operation
  except subnormal results: at the onset of the Ricker wavelet (values
  down to 1e-45) their fixed absolute rounding differs between the two runs,
  and the time stepping carries those differences into the signal (the CPU
  oracle shows the same, 4e-6 on the 80x60 model): relative L2 <= 5e-5, at
  the full sizes of the coupled 400x200 model (4000 steps), the batched
  1000x500 GRF model (32 shots) and the 3D 128x128x64 model;
* superposition: two sources in one run equal the sum of two one-source runs
  to FP32 precision, relative L2 <= 5e-5 (coupled 400x200, 4000 steps);
* finiteness and non-trivial signal everywhere.
"""
from dataclasses import replace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run2d(w, srcs, nstep, nshots=1, **kw):
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=nstep, nshots=nshots, **kw)
    sim.set_sources(srcs)
    sim.set_receivers(w.rec_x, w.rec_z)
    sim.initialize()
    sim.run(nstep)
    assert sim.check_finite()
    return sim.seismograms()


def test_coupled_400x200_linearity_and_superposition(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.coupled_400x200()
    s0 = w.sources[0]
    a = run2d(w, [s0], w.nstep)
    b = run2d(w, [replace(s0, factor=2 * s0.factor)], w.nstep)
    assert np.abs(a).max() > 0
    assert rel(b, 2 * a) <= 5e-5
    # same f0 (and no shift): both runs share the start time t0 = -1.2/f0
    s1 = replace(s0, x=s0.x + 3100.0, z=s0.z - 700.0, factor=0.5 * s0.factor)
    c = run2d(w, [s1], w.nstep)
    both = run2d(w, [s0, s1], w.nstep)
    assert np.linalg.norm(both - (a + c)) <= 5e-5 * np.linalg.norm(both)


def test_batched_1000x500_linearity(sfg_lib):
    from specfempp_b200 import meshgen
    w = meshgen.elastic_grf_1000x500(nstep=3000, nshots=32)
    kw = dict(point_rho=w.point_rho, point_vp=w.point_vp, point_vs=w.point_vs)
    a = run2d(w, w.sources, 3000, nshots=32, **kw)
    b = run2d(w, [replace(s, factor=2 * s.factor) for s in w.sources], 3000, nshots=32, **kw)
    # the nearer sources' waves reach the receiver line within the 1.5 s
    assert (np.abs(a).reshape(32, -1).max(axis=1) > 1e-12).sum() >= 8
    assert rel(b, 2 * a) <= 5e-5


def test_elastic3d_128x128x64_linearity(sfg_lib):
    from specfempp_b200 import meshgen, sfg3d
    w = meshgen.elastic3d_layered_grf(nstep=300)
    out = []
    for scale in (1.0, 2.0):
        sim = sfg3d.Simulation3D(w.mesh, dt=w.dt, nstep=300)
        sim.set_sources([replace(s, factor=scale * s.factor) for s in w.sources])
        sim.set_receivers(w.rec_xyz)
        sim.initialize()
        sim.run(300)
        assert sim.check_finite()
        out.append(sim.seismograms())
        sim.close()
    assert np.abs(out[0]).max() > 0
    assert rel(out[1], 2 * out[0]) <= 5e-5
