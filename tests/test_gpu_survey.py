"""Shot sharding with the real library: two processes, each with its own
Simulation2D on the GPU, gloo collectives between them.

The survey helpers (specfempp_b200.survey) must give what one process gives
for the whole survey: the gathered seismograms of every shot (the same bits:
the forward kernels are deterministic), and the summed L2 misfit and rho /
kappa / mu gradient of every source (to FP32 round-off: each process times
the launch shape of its reverse kernels itself, and the float64 sum over
sources runs in another order).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

NX, NZ, NSTEP, INTERVAL, NSRC = 60, 30, 240, 40, 5


def workload():
    from specfempp_b200 import adjoint, meshgen
    aw = meshgen.elastic_adjoint_500x250(nstep=NSTEP, nx=NX, nz=NZ, nsrc=NSRC, nrec=12)
    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731
    kt, mt = adjoint.moduli(f64(aw.true_rho), f64(aw.true_vp), f64(aw.true_vs))
    w = aw.workload
    k0, m0 = adjoint.moduli(f64(w.point_rho), f64(w.point_vp), f64(w.point_vs))
    return aw, (f64(aw.true_rho), kt, mt), (f64(w.point_rho), k0, m0)


def make_sim(w):
    from specfempp_b200 import sfg
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=NSTEP, point_rho=w.point_rho, point_vp=w.point_vp,
                           point_vs=w.point_vs)
    sim.set_sources([w.sources[0]])
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    return sim


def _worker(rank, world, port, outdir):
    import torch
    import torch.distributed as dist

    from specfempp_b200 import adjoint, survey
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        aw, true_m, m0 = workload()
        w = aw.workload
        sim = make_sim(w)
        obs = adjoint.observed_data(sim, w.sources, *true_m, NSTEP)
        # the traces of this rank's shots, gathered in shot order
        mine = survey.shard(NSRC, world, rank)
        local = obs[list(mine)].astype(np.float32)
        full = survey.gather_seismograms(local, NSRC)
        L, g = survey.distributed_l2_gradient(sim, w.sources, *m0, obs, NSTEP, INTERVAL)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), L=L, g0=g[0], g1=g[1], g2=g[2], full=full, obs=obs)
        sim.close()
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_processes_on_real_simulations_match_one_process(tmp_path, sfg_lib):
    from specfempp_b200 import adjoint
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    aw, true_m, m0 = workload()
    w = aw.workload
    sim = make_sim(w)
    obs = adjoint.observed_data(sim, w.sources, *true_m, NSTEP)
    L1, g1 = adjoint.l2_misfit_gradient(sim, w.sources, *m0, obs, NSTEP, INTERVAL)
    assert L1 > 0
    for r in range(2):
        z = np.load(os.path.join(tmp_path, f"r{r}.npz"))
        assert np.array_equal(z["obs"], obs)                       # same bits in every process
        assert np.array_equal(z["full"], obs.astype(np.float32))   # gathered in shot order
        assert np.isclose(float(z["L"]), L1, rtol=1e-12)
        for k in range(3):
            assert np.linalg.norm(z[f"g{k}"] - g1[k]) <= 1e-5 * np.linalg.norm(g1[k]), k
