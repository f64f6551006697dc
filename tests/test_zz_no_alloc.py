"""sfg_step_noalloc: one time step that allocates no device memory.

Some callers cannot call cudaMalloc while they step: a host framework that
owns and budgets all device memory itself, or a time loop that runs after
the device memory has been sized and frozen.  For them the library offers a
step that works on the caller's own field buffers and keeps its only scratch
(the element kernel's accumulator) in a fixed array inside the library.

These tests call it through the C ABI and check that two calls in a row give
the same fields as the handle-based sfg_step from the same state, within the
1e-5 relative L2 used by the other parity tests, and that a model larger than
the fixed scratch is refused.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _handle(w):
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep)
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_x, w.rec_z)
    sim.initialize()
    return sim


def test_noalloc_step_matches_sfg_step(sfg_lib):
    import torch
    from specfempp_b200 import meshgen

    w = meshgen.elastic_psv_80x60(nstep=330)
    sim = _handle(w)
    k = 300                                   # a developed wavefield, with Stacey and the source
    sim.run(k)
    start = {f: sim.field("elastic", f).copy() for f in ("displacement", "velocity", "acceleration")}
    expected = []
    for _ in range(2):
        sim.step()
        expected.append({f: sim.field("elastic", f).copy()
                         for f in ("displacement", "velocity", "acceleration")})

    dev = torch.device("cuda", 0)
    u = torch.from_numpy(start["displacement"]).to(dev).contiguous()
    v = torch.from_numpy(start["velocity"]).to(dev).contiguous()
    a = torch.from_numpy(start["acceleration"]).to(dev).contiguous()
    torch.cuda.synchronize()
    for call in range(2):
        rc = sfg_lib.sfg_step_noalloc(sim.h, k + call, C.c_void_p(u.data_ptr()),
                                      C.c_void_p(v.data_ptr()), C.c_void_p(a.data_ptr()))
        assert rc == 0, sfg_lib.sfg_last_error(sim.h)
        got = {"displacement": u.cpu().numpy(), "velocity": v.cpu().numpy(),
               "acceleration": a.cpu().numpy()}
        for f, ref in expected[call].items():
            assert np.all(np.isfinite(got[f]))
            assert rel_l2(got[f], ref) <= 1e-5, (call, f, rel_l2(got[f], ref))
    # the handle's own state is untouched by the no-allocation calls
    assert np.array_equal(sim.field("elastic", "displacement"), expected[1]["displacement"])


def test_noalloc_refuses_models_above_the_scratch(sfg_lib):
    import torch
    from specfempp_b200 import meshgen

    # 600 x 300 quads: 2,883,601 two-component points, above the 2,097,152 limit
    w = meshgen.elastic_grf_1000x500(nstep=4, nshots=1, nrec=2, nx=600, nz=300)
    w.point_rho = w.point_vp = w.point_vs = None
    sim = _handle(w)
    n = sim.info().nglob_elastic * 2
    buf = torch.zeros(3, n, device="cuda")
    rc = sfg_lib.sfg_step_noalloc(sim.h, 0, C.c_void_p(buf[0].data_ptr()),
                                  C.c_void_p(buf[1].data_ptr()), C.c_void_p(buf[2].data_ptr()))
    assert rc == -1
    assert b"fixed scratch" in sfg_lib.sfg_last_error(sim.h)


def test_noalloc_reports_a_nonfinite_step(sfg_lib):
    import torch
    from specfempp_b200 import meshgen

    w = meshgen.elastic_psv_80x60(nstep=8)
    sim = _handle(w)
    n = sim.info().nglob_elastic * 2
    buf = torch.zeros(3, (n + 3) // 4 * 4, device="cuda")   # rows on 16-byte boundaries
    buf[0, 7] = float("nan")                  # a blown-up displacement
    torch.cuda.synchronize()
    rc = sfg_lib.sfg_step_noalloc(sim.h, 0, C.c_void_p(buf[0].data_ptr()),
                                  C.c_void_p(buf[1].data_ptr()), C.c_void_p(buf[2].data_ptr()))
    assert rc == -6, sfg_lib.sfg_last_error(sim.h)
    assert b"NaN" in sfg_lib.sfg_last_error(sim.h)
    # a clean state steps again with SFG_OK: the flag is cleared per call
    buf.zero_()
    torch.cuda.synchronize()
    rc = sfg_lib.sfg_step_noalloc(sim.h, 1, C.c_void_p(buf[0].data_ptr()),
                                  C.c_void_p(buf[1].data_ptr()), C.c_void_p(buf[2].data_ptr()))
    assert rc == 0, sfg_lib.sfg_last_error(sim.h)


def test_noalloc_refuses_misaligned_fields_before_any_launch(sfg_lib):
    import torch
    from specfempp_b200 import meshgen

    w = meshgen.elastic_psv_80x60(nstep=8)
    sim = _handle(w)
    n = sim.info().nglob_elastic * 2
    buf = torch.zeros(3 * n + 8, device="cuda")
    u = buf[1:1 + n]                          # 4 bytes past a 16-byte boundary
    v = buf[n + 4:2 * n + 4]
    a = buf[2 * n + 4:3 * n + 4]
    rc = sfg_lib.sfg_step_noalloc(sim.h, 0, C.c_void_p(u.data_ptr()), C.c_void_p(v.data_ptr()),
                                  C.c_void_p(a.data_ptr()))
    assert rc == -1
    assert b"16-byte" in sfg_lib.sfg_last_error(sim.h)
    torch.cuda.synchronize()
    assert torch.count_nonzero(buf).item() == 0   # nothing ran
