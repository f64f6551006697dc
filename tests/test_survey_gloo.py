"""Shot sharding across processes (gloo, world size 2, CPU): the survey
helpers give the same misfit, gradient and gathered traces as one process."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

NSTEP, NREC, SHAPE = 12, 3, (4, 25)


class FakeSim:
    """Deterministic stand-in for Simulation2D's adjoint interface (no GPU)."""

    def set_model(self, rho, kappa, mu):
        self.m = (np.asarray(rho, np.float64), np.asarray(kappa, np.float64), np.asarray(mu, np.float64))

    def set_sources(self, srcs):
        (self.s,) = srcs

    def forward_checkpointed(self, nsteps, interval):
        t = np.arange(nsteps)[:, None, None]
        return np.sin(0.3 * t + self.s.x + np.arange(NREC)[None, :, None] + np.arange(2)) * self.m[0].mean()

    def adjoint_gradient(self, res):
        w = float(np.asarray(res).sum()) + self.s.x
        return tuple((k + 1.0) * w * m / m.sum() for k, m in enumerate(self.m))


class Src:
    def __init__(self, x):
        self.x = x


def sources():
    return [Src(0.1 * i) for i in range(5)]


def model():
    rng = np.random.default_rng(0)
    return [1.0 + rng.random(SHAPE) for _ in range(3)]


def observed():
    return np.stack([np.cos(0.1 * np.arange(NSTEP))[:, None, None] * np.ones((NREC, 2)) * i for i in range(5)])


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from specfempp_b200 import survey
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        L, g = survey.distributed_l2_gradient(FakeSim(), sources(), *model(), observed(), NSTEP, 4)
        mine = survey.shard(7, world, rank)
        local = np.stack([np.full((NSTEP, NREC, 2), float(i)) for i in mine]).astype(np.float32)
        full = survey.gather_seismograms(local, 7)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), L=L, g0=g[0], g1=g[1], g2=g[2], full=full)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_and_balances():
    from specfempp_b200 import survey
    for n in (0, 1, 5, 7, 32):
        for world in (1, 2, 3, 8):
            parts = [list(survey.shard(n, world, r)) for r in range(world)]
            assert sum(parts, []) == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        survey.shard(4, 2, 2)


def test_two_rank_gradient_and_gather_match_one_process(tmp_path):
    from specfempp_b200 import adjoint
    mp.spawn(_worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    L1, g1 = adjoint.l2_misfit_gradient(FakeSim(), sources(), *model(), observed(), NSTEP, 4)
    for r in range(2):
        z = np.load(os.path.join(tmp_path, f"r{r}.npz"))
        assert np.isclose(float(z["L"]), L1, rtol=1e-12)
        for k in range(3):
            assert np.allclose(z[f"g{k}"], g1[k], rtol=1e-12)
        assert np.array_equal(z["full"][:, 0, 0, 0], np.arange(7, dtype=np.float32))
