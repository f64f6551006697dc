"""Shots across GPUs: one process per GPU, shots (sources) are independent.

The time loop of one shot has no exchange step, so a survey shards by shot
with no collective inside the time loop:

* ``shard``: the contiguous block of shots a rank owns;
* ``gather_seismograms``: every rank's traces of its shots, concatenated in
  shot order (all-gather over the process group after the runs);
* ``distributed_l2_gradient``: the waveform misfit and its gradient summed
  over all sources, each rank running the adjoint of its own sources and one
  all-reduce (sum) of (misfit, d/drho, d/dkappa, d/dmu) at the end — the
  reference's adjoint workflow sums event kernels the same way.

The process group is ``torch.distributed``'s (NCCL on GPUs, gloo on CPU);
tensors are moved to the group's device for the collectives.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def shard(n: int, world: int, rank: int) -> range:
    """Balanced contiguous block of range(n) for `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _device(group=None):
    backend = dist.get_backend(group)
    return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def gather_seismograms(local: np.ndarray, nshots: int, group=None) -> np.ndarray:
    """Concatenate each rank's [its shots, ...] array in shot order."""
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    mine = shard(nshots, world, rank)
    if local.shape[0] != len(mine):
        raise ValueError("local array does not hold this rank's shots")
    per = max(len(shard(nshots, world, r)) for r in range(world))
    dev = _device(group)
    buf = torch.zeros((per,) + local.shape[1:], dtype=torch.float64, device=dev)
    buf[: len(mine)] = torch.from_numpy(np.asarray(local, np.float64)).to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = [parts[r][: len(shard(nshots, world, r))].cpu().numpy() for r in range(world)]
    return np.concatenate(out).astype(local.dtype)


def distributed_l2_gradient(sim, sources, rho, kappa, mu, observed, nsteps: int, interval: int, group=None):
    """Misfit and gradient over all sources; this rank runs its shard.

    ``observed``: [nsrc, nsteps, nrec, 2] for all sources (each rank reads
    only its own).  Returns (misfit, (d/drho, d/dkappa, d/dmu)) summed over
    every rank, identical on all ranks."""
    from . import adjoint
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    mine = list(shard(len(sources), world, rank))
    shape = np.shape(rho)
    if mine:
        L, g = adjoint.l2_misfit_gradient(sim, [sources[i] for i in mine], rho, kappa, mu,
                                          np.asarray(observed)[mine], nsteps, interval)
    else:
        L, g = 0.0, tuple(np.zeros(shape) for _ in range(3))
    dev = _device(group)
    flat = torch.from_numpy(np.concatenate([[L]] + [np.asarray(x, np.float64).ravel() for x in g])).to(dev)
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat = flat.cpu().numpy()
    n = int(np.prod(shape))
    grads = tuple(flat[1 + k * n: 1 + (k + 1) * n].reshape(shape) for k in range(3))
    return float(flat[0]), grads
