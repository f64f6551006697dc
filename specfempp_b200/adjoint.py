"""Model gradients of seismograms through the discrete adjoint (2D isotropic
elastic P-SV and SH).

``SeismogramFunction`` is a ``torch.autograd.Function`` whose forward runs the
library's checkpointed forward simulation for a per-GLL-point model
(rho, kappa, mu), and whose backward runs the library's reverse sweep
(``sfg_adjoint_gradient``): the exact adjoint of the FP32 time step, so that
``loss.backward()`` yields dL/drho, dL/dkappa, dL/dmu per GLL point.

It plays the part of the reference's adjoint workflow — a forward run that
stores the wavefield (include/io/wavefield/writer.tpp), a combined
adjoint/backward run (core/specfem/solver/time_marching.tpp:133-264) and the
Frechet kernels (include/medium/dim2/elastic/isotropic/frechet_derivative.hpp)
— with checkpoints kept in HBM instead of a wavefield file.  The Stacey
impedances (rho vp, rho vs) are differentiated with the rest of the model,
so the gradient is exact on the absorbing edges too (the reference's
kernels carry no boundary term).  In SH the gradient with respect to kappa
is zero.
"""
from __future__ import annotations

import numpy as np
import torch

from .sfg import Simulation2D


class SeismogramFunction(torch.autograd.Function):
    """seis[nsteps, nrec, 2] = F(rho, kappa, mu) for a prepared simulation."""

    @staticmethod
    def forward(ctx, rho, kappa, mu, sim: Simulation2D, nsteps: int, interval: int):
        sim.set_model(*(t.detach().to("cpu", torch.float32).numpy() for t in (rho, kappa, mu)))
        seis = sim.forward_checkpointed(nsteps, interval)
        ctx.sim = sim
        ctx.dtype = rho.dtype
        ctx.device = rho.device
        return torch.from_numpy(np.ascontiguousarray(seis)).to(rho.device)

    @staticmethod
    def backward(ctx, grad_seis):
        g = grad_seis.detach().to("cpu", torch.float32).contiguous().numpy()
        grho, gkappa, gmu = ctx.sim.adjoint_gradient(g)
        out = [torch.from_numpy(x).to(ctx.device, ctx.dtype) for x in (grho, gkappa, gmu)]
        return out[0], out[1], out[2], None, None, None


def seismograms(sim: Simulation2D, rho, kappa, mu, nsteps: int, interval: int = 100):
    """Differentiable displacement seismograms [nsteps, nrec, 2] of ``sim``.

    ``sim`` must be initialised with one elastic P-SV medium, one shot and
    displacement receivers sampled every step; rho, kappa, mu are tensors of
    shape [nspec, 25] (database element order).  ``interval`` is the number
    of steps between checkpoints: device memory is 3 states per checkpoint
    plus 2 states per step of one interval.
    """
    return SeismogramFunction.apply(rho, kappa, mu, sim, int(nsteps), int(interval))


def moduli(rho, vp, vs):
    """(kappa, mu) of the reference's elastic isotropic material:
    mu = rho vs^2, kappa = rho (vp^2 - 4/3 vs^2)
    (include/medium/dim2/elastic/isotropic/material.hpp:66-69)."""
    mu = rho * vs * vs
    return rho * vp * vp - 4.0 / 3.0 * mu, mu


def l2_misfit_gradient(sim: Simulation2D, sources, rho, kappa, mu, observed, nsteps: int,
                       interval: int):
    """Waveform misfit L = sum over sources of 1/2 ||d_s - d_obs,s||^2 and its
    gradient (dL/drho, dL/dkappa, dL/dmu) per GLL point [nspec, 25].

    ``observed``: [nsrc, nsteps, nrec, 2].  Each source runs as the handle's
    single source in turn (forward with checkpoints, then the adjoint with the
    residual as adjoint source), and the gradients are summed, as the
    reference's adjoint workflow sums event kernels.
    """
    sim.set_model(rho, kappa, mu)
    total = 0.0
    grads = [np.zeros(np.shape(rho), np.float64) for _ in range(3)]
    for s, src in enumerate(sources):
        sim.set_sources([src])
        syn = sim.forward_checkpointed(nsteps, interval).astype(np.float64)
        res = syn - np.asarray(observed[s], np.float64)
        total += 0.5 * float((res * res).sum())
        g = sim.adjoint_gradient(res.astype(np.float32))
        for a, b in zip(grads, g):
            a += b
    return total, tuple(grads)


def l2_misfit(sim: Simulation2D, sources, rho, kappa, mu, observed, nsteps: int) -> float:
    """The misfit of ``l2_misfit_gradient`` without the gradient (forward runs only)."""
    sim.set_model(rho, kappa, mu)
    total = 0.0
    for s, src in enumerate(sources):
        sim.set_sources([src])
        syn = _forward(sim, nsteps).astype(np.float64)
        res = syn - np.asarray(observed[s], np.float64)
        total += 0.5 * float((res * res).sum())
    return total


def observed_data(sim: Simulation2D, sources, rho, kappa, mu, nsteps: int) -> np.ndarray:
    """Displacement seismograms [nsrc, nsteps, nrec, 2] of a model (the 'true' data)."""
    sim.set_model(rho, kappa, mu)
    out = []
    for src in sources:
        sim.set_sources([src])
        out.append(_forward(sim, nsteps))
    return np.stack(out)


def _forward(sim: Simulation2D, nsteps: int) -> np.ndarray:
    sim.reset()
    sim.run(nsteps)
    return sim.seismograms()[0, :nsteps, 0].copy()
