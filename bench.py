"""Benchmark of the spectral-element time step (GLL-point updates per second).

Workload: the coupled acoustic-elastic 2D model (400x200 quads over 20x10 km,
NGLL=5, 1,282,401 global GLL points, 1.5 km of water over 4 seeded elastic
layers, Stacey on three sides, acoustic free surface on top, Ricker 5 Hz
pressure source, 200 seafloor receivers, dt = 1e-3 s).  Synthetic, seeded.

One bench step = one time step of the whole model.  Reported keys:
* value:  GLL-point updates/s with inputs resident in HBM, every timed step
          launched after an L2 flush (a 256 MiB write, then a read of another
          256 MiB buffer: no input and no dirty line left in the cache), timed
          with CUDA events on the handle's stream, summed over the K steps,
          max over ranks;
* e2e:    the same metric through the per-step C-ABI call with host buffers
          (STF row host->device, seismogram row device->host, a sync per step);
* roofline: the dominant kernel (the element kernel of one step: one
          owner-computes launch, or the colour passes, whichever the autotuner
          chose) against the measured HBM bandwidth, its launch timed after the
          same L2 flush (frac) and back to back (frac_back_to_back);
* cpu_baseline: the CPU oracle (a C++ restatement of the reference) on all
          host cores, a bounded sample of the same workload sized by a short
          probe run to about CPU_SAMPLE_S (10 s) of CPU time.
``--impl reference`` times that CPU implementation alone on the same
workload and metric.  With --gpus N > 1 every rank runs an independent
replica (the single-shot path does not shard) and value sums the ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GLL-point updates/s"
UNIT = "GLL-pt/s"
WORKLOAD = "coupled_400x200"
# algorithmic bytes of the elastic stiffness kernel: per element GLL point
# ibool(4) + xix,xiz,gammax,gammaz,|J| (20) + lambda+2mu, mu (8) = 32 B; per
# elastic global point u read (8) + accumulator read and write (16) = 24 B.
STIFF_B_PER_LOCAL = 32
STIFF_B_PER_GLOB = 24
# acoustic element point: ibool + Jacobian (20) + 1/rho = 28 B; point: chi read,
# accumulator read and write = 12 B
STIFF_B_PER_LOCAL_AC = 28
STIFF_B_PER_GLOB_AC = 12
# whole step, per global point (2D elastic P-SV, FP32): u,v,a read+write 48 +
# M^-1 8 + 32 B per local point x 25 nspec / nglob.
FLUSH_BYTES = 256 << 20       # L2 flush before every timed step (the L2 is 126 MB)
STEP_B_GLOB = 56
STEP_B_LOCAL = 32


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile():
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, device_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap,power.draw")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device_index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for k, n in enumerate(names):
                    if r[2 + k].strip().lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(mx)) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(name, nstep):
    from specfempp_b200 import meshgen
    if name == "coupled_400x200":
        return meshgen.coupled_400x200(nstep=nstep)
    if name == "elastic_psv_80x60":
        return meshgen.elastic_psv_80x60(nstep=nstep)
    raise SystemExit(f"unknown workload {name}")


def workload_config(name, w, nglob):
    """The config dict of both arms (GPU and --impl reference): the workload
    only, so that the two lines describe the same run."""
    mesh = w.mesh
    med = np.asarray(mesh.mat_medium)[np.asarray(mesh.kmato)]
    nel = int((med == 1).sum())
    return {"workload": name, "nglob": int(nglob), "nspec": int(mesh.nspec), "nspec_elastic": nel,
            "nspec_acoustic": int(mesh.nspec) - nel, "dt": w.dt, "ngll": 5, "shots": 1,
            "l2": "flushed before every timed step (256 MiB written, then another 256 MiB read, "
                  "outside the timed interval: the cache holds no input and no dirty line)"}


CPU_SAMPLE_S = 10.0   # seconds of CPU work per baseline sample (a short probe sizes it)


def sample_steps(probe_steps, probe_seconds, cap):
    """Steps for about CPU_SAMPLE_S seconds of oracle time, from a probe run."""
    per = max(probe_seconds / max(probe_steps, 1), 1e-6)
    return int(min(cap, max(probe_steps, math.ceil(CPU_SAMPLE_S / per))))


def cpu_oracle_throughput(w, steps, threads):
    from oracle import runner
    case = runner.Case2D(mesh=w.mesh, sources=w.sources, rec_x=w.rec_x, rec_z=w.rec_z, dt=w.dt,
                         nstep=steps)
    r = runner.run(case, "f32", nthreads=threads)
    return r["nglob"] * steps / r["loop_seconds"], r["loop_seconds"]


def bench_batched(args, world, barrier, max_over_ranks):
    """Config 3: S shots on a 2D elastic GRF model, batched in one launch per
    step against the same shots run one at a time (shot.steps/s).  The model
    holds S x 8M points of state (inputs far larger than L2); timed with CUDA
    events over graph-replayed steps.  With N ranks the survey of S shots is
    sharded, S/N shots per rank (strong scaling of one survey, no collective
    during the time loop; timings are the max over ranks)."""
    from specfempp_b200 import meshgen, sfg, survey
    nx, nz = (int(v) for v in args.batched_mesh.split("x"))
    S_total = args.batched_shots
    rank = int(os.environ.get("RANK", "0"))
    mine = list(survey.shard(S_total, world, rank))
    S = len(mine)
    steps = args.batched_steps
    warm = 3
    wall = meshgen.elastic_grf_1000x500(nstep=steps + warm + 2, nshots=S_total, nx=nx, nz=nz)
    from dataclasses import replace as _replace
    w = _replace(wall, sources=[_replace(s, shot=mine.index(s.shot)) for s in wall.sources if s.shot in mine])

    def make(nshots, srcs):
        sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep, nshots=nshots, point_rho=w.point_rho,
                               point_vp=w.point_vp, point_vs=w.point_vs,
                               kernel_variant=args.batched_variant if nshots > 1 else 0)
        sim.set_sources(srcs)
        sim.set_receivers(w.rec_x, w.rec_z)
        sim.initialize()
        return sim

    sim = make(S, w.sources)
    inf = sim.info()
    sim.run(warm)
    barrier()
    ms_b = max_over_ranks(sim.run_timed(steps))
    variant = inf.kernel_variant
    if variant == 5:
        # fused tile kernel (elements + interior points) and the boundary points
        kern = {"batched_tile_kernel_ms": sim.time_kernel(0, 5), "batched_boundary_ms": sim.time_kernel(1, 5)}
    else:
        kern = {"batched_stiffness_ms": sim.time_kernel(0, 5)}
    del sim
    from dataclasses import replace
    one = make(1, [replace(w.sources[0], shot=0)])
    one.run(warm)
    barrier()
    ms_1 = max_over_ranks(one.run_timed(steps))
    del one
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        # the reference runs one shot at a time: 50 steps of one shot on the
        # host cores (oracle, FP32, full mesh and model)
        from oracle import runner
        threads = os.cpu_count() or 1

        def one_shot(n):
            case = runner.Case2D(mesh=w.mesh, sources=[replace(w.sources[0], shot=0)], rec_x=w.rec_x,
                                 rec_z=w.rec_z, dt=w.dt, nstep=n, point_rho=w.point_rho, point_vp=w.point_vp,
                                 point_vs=w.point_vs)
            return runner.run(case, "f32", nthreads=threads)["loop_seconds"]
        n = sample_steps(10, one_shot(10), 3000)
        secs = one_shot(n)
        cpu = {"value": n / secs, "unit": "shot-steps/s", "cores": threads, "kind": "port",
               "sample": f"{n} time steps of one shot of elastic_grf_{nx}x{nz}, FP32 C++ restatement of the "
                         f"reference on {threads} host threads ({secs:.2f} s)"}
    rate_b = S_total * steps / (ms_b / 1e3)
    rate_1 = world * steps / (ms_1 / 1e3)
    per_shot_b = STEP_B_GLOB + STEP_B_LOCAL * inf.nspec * 25 / (inf.nglob * S)
    return {"workload": f"elastic_grf_{nx}x{nz}", "shots": S_total, "shots_per_gpu": S, "nglob": inf.nglob,
            "scaling": "strong (one survey of the shots, sharded by shot)",
            "steps": steps, "ms_per_step_batched": ms_b / steps, "ms_per_step_one_shot": ms_1 / steps,
            "shot_steps_per_s_batched": rate_b, "shot_steps_per_s_one_at_a_time": rate_1,
            "speedup": rate_b / rate_1,
            "gll_pt_updates_per_s_batched": rate_b * inf.nglob,
            "kernel_variant": variant, **kern,
            "batched_frac_of_hbm": per_shot_b * inf.nglob * S / (ms_b / steps / 1e3) / 1e9 / peaks()[0],
            "timing": "CUDA events, graph-replayed steps, inputs larger than L2",
            "cpu_baseline": cpu}


def bench_adjoint(args, world, barrier, max_over_ranks):
    """Config 4: cost of the L2-misfit gradient of all the configuration's
    sources (per source a checkpointed forward, the segment recompute and the
    reverse sweep; the gradients summed) against plain forward runs of the
    same sources, on the 500x250 elastic model (wall clock around synchronous
    calls, after one untimed gradient that allocates the checkpoints and
    captures the recording graphs).  With --adjoint-fd K (default 8), also
    the fourth-order central-difference check of that gradient along K
    seeded smooth perturbations; the error of a direction is measured
    against the largest directional derivative of the set, because a
    direction that misses the wave paths has a derivative at the FP32
    noise floor of the difference quotient."""
    from specfempp_b200 import adjoint, meshgen, sfg
    nx, nz = (int(v) for v in args.adjoint_mesh.split("x"))
    nstep = args.adjoint_steps
    aw = meshgen.elastic_adjoint_500x250(nstep=nstep, nx=nx, nz=nz)
    w = aw.workload
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=nstep, point_rho=w.point_rho, point_vp=w.point_vp,
                           point_vs=w.point_vs)
    sim.set_sources([w.sources[0]])
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    inf = sim.info()
    f64 = lambda a: a.astype(np.float64)  # noqa: E731
    kt, mt = adjoint.moduli(f64(aw.true_rho), f64(aw.true_vp), f64(aw.true_vs))
    rho0 = f64(w.point_rho)
    k0, m0 = adjoint.moduli(rho0, f64(w.point_vp), f64(w.point_vs))
    srcs = w.sources
    obs = adjoint.observed_data(sim, srcs, aw.true_rho, kt, mt, nstep)
    sim.set_model(rho0, k0, m0)

    def forward_s():
        barrier()
        t0 = time.perf_counter()
        for src in srcs:
            sim.set_sources([src])
            sim.reset()
            sim.run(nstep)
            sim.synchronize()
        return time.perf_counter() - t0

    def gradient_s():
        barrier()
        t0 = time.perf_counter()
        L, g = adjoint.l2_misfit_gradient(sim, srcs, rho0, k0, m0, obs, nstep, aw.interval)
        return time.perf_counter() - t0, L, g

    forward_s()
    _, L, grads = gradient_s()
    t_fwd = max_over_ranks(min(forward_s() for _ in range(2)))
    t_grad = max_over_ranks(min(gradient_s()[0] for _ in range(2)))
    out = {"workload": f"elastic_adjoint_{nx}x{nz}", "nglob": inf.nglob, "steps": nstep,
           "sources": len(srcs), "checkpoint_interval": aw.interval,
           "segments": -(-nstep // aw.interval), "segments_kept_from_forward": sim.adjoint_buffers(),
           "segment_budget": "default: 75% of the free device memory", "forward_s": t_fwd,
           "gradient_s": t_grad, "cost_ratio": t_grad / t_fwd,
           "gradient_gll_pt_steps_per_s": inf.nglob * nstep * len(srcs) / t_grad,
           "timing": "wall clock around synchronous calls; forward = plain runs of every source; "
                     "gradient = per source checkpointed forward (recording the segments the buffers "
                     "hold) + recompute of the other segments + reverse sweep"}
    if args.adjoint_fd > 0:
        xmax, zmax = 25.0 * nx, 25.0 * nz
        pert = meshgen.smooth_perturbations(w.mesh, xmax, zmax, args.adjoint_fd, 1000.0, seed=7)
        model = [rho0, k0, m0]
        rows = []
        h = 0.02
        for i in range(args.adjoint_fd):
            which = i % 3
            d = pert[i] * model[which]

            def f(hh):
                m = [x.copy() for x in model]
                m[which] = m[which] + hh * d
                return adjoint.l2_misfit(sim, srcs, *m, obs, nstep)
            fd = (8.0 * (f(h) - f(-h)) - (f(2 * h) - f(-2 * h))) / (12.0 * h)
            ad = float((grads[which] * d).sum())
            rows.append({"parameter": ["rho", "kappa", "mu"][which], "adjoint": ad, "fd4": fd,
                         "rel_err": abs(ad - fd) / abs(fd)})
        scale = max(abs(r["fd4"]) for r in rows)
        for r in rows:
            r["err_vs_largest"] = abs(r["adjoint"] - r["fd4"]) / scale
        worst = max(r["err_vs_largest"] for r in rows)
        out["fd"] = {"misfit": L, "sources": len(srcs), "step": h, "stencil": "4th-order central",
                     "perturbations": rows, "max_rel_err": max(r["rel_err"] for r in rows),
                     "max_err_vs_largest_derivative": worst,
                     "criterion": "max over directions of |adjoint - fd4| / max |fd4| <= 1e-3",
                     "pass": bool(worst <= 1e-3)}
    del sim
    return out


def bench_3d(args, world, barrier, max_over_ranks):
    """Config 5: 3D elastic hexahedral mesh (128x128x64 elements over 64x64x32 km,
    67,634,433 global GLL points), layered background + 5% GRF, free top and
    Stacey on the other faces, moment tensor (1 Hz), 1000 surface receivers,
    dt = 2 ms.  A bounded run of the 5000-step configuration: 10 warm-up steps,
    then K steps back to back (CUDA events, graph replay) and K steps each after
    a 256 MiB L2 flush; model state (about 12.6 GB) far larger than L2."""
    from specfempp_b200 import meshgen, sfg3d
    nx, ny, nz = (int(v) for v in args.mesh3d.split("x"))
    steps = args.steps3d
    t0 = time.perf_counter()
    w = meshgen.elastic3d_layered_grf(nx, ny, nz, nstep=2 * steps + 20, nrec=1000)
    sim = sfg3d.Simulation3D(w.mesh, dt=w.dt, nstep=w.nstep, elements_per_block=args.epb3d)
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_xyz, types=("displacement",))
    sim.initialize()
    setup_s = time.perf_counter() - t0
    inf = sim.info()
    sim.run(10)
    barrier()
    ms_b2b = max_over_ranks(sim.run_timed(steps))
    ms_fl = max_over_ranks(sim.run_timed_flushed(steps))
    stiff = sim.time_kernel(0, 10)
    upd = sim.time_kernel(1, 10)
    finite = sim.check_finite()
    r = 125.0 * inf.nspec / inf.nglob
    alg = 84.0 + 52.0 * r                       # algorithmic bytes per point-step
    peak, _ = peaks()
    out = {"workload": f"elastic3d_{nx}x{ny}x{nz}", "nglob": inf.nglob, "nspec": inf.nspec,
           "elements_per_block": inf.elements_per_block, "kernel_variant": inf.kernel_variant,
           "steps": steps, "setup_s": setup_s,
           "device_gb": inf.device_bytes / 1e9,
           "ms_per_step_flushed": ms_fl / steps, "ms_per_step_back_to_back": ms_b2b / steps,
           "gll_pt_updates_per_s": world * inf.nglob * steps / (ms_fl / 1e3),
           "gll_pt_updates_per_s_back_to_back": world * inf.nglob * steps / (ms_b2b / 1e3),
           "element_kernel_ms": stiff, "update_kernel_ms": upd,
           "algorithmic_bytes_per_point": alg,
           "step_frac_of_hbm": alg * inf.nglob / (ms_fl / steps / 1e3) / 1e9 / peak,
           "finite": bool(finite)}
    sim.close()
    rank = int(os.environ.get("RANK", "0"))
    if world == 1 and not args.no_cpu_baseline:
        # a bounded sample: 5 steps of the full 67.6 M-point model on the host
        # cores (the oracle's 3D restatement, FP32)
        from oracle import runner3d
        threads = os.cpu_count() or 1

        def run3d(n):
            return runner3d.run(runner3d.Case3D(w.mesh, w.sources, w.rec_xyz, w.dt, n), "f32",
                                nthreads=threads)["loop_seconds"]
        n = sample_steps(2, run3d(2), 200)
        secs = run3d(n)
        out["cpu_baseline"] = {"value": inf.nglob * n / secs, "unit": "GLL-pt/s", "cores": threads,
                               "kind": "port",
                               "sample": f"{n} time steps of elastic3d_{nx}x{ny}x{nz}, FP32 C++ restatement of the "
                                         f"reference on {threads} host threads ({secs:.2f} s)"}
    return out


def bench_media(args, world, barrier, max_over_ranks):
    """Throughput of the other media on fixed synthetic meshes (seeded, no
    dataset): a 400 x 400 porous block over 10 x 10 km (four components,
    viscous pore fluid, layered), and an acoustic-elastic model with a nonconforming interface
    (400 elastic columns under 600 water columns, 200 + 150 rows).  10
    warm-up steps, then K steps after a 256 MiB L2 flush each and K steps
    back to back (CUDA events, graph replay).  Algorithmic bytes per
    poroelastic point-step: read u, v, a and M^-1 (4 components) and write
    u, v, a = 112 B per global point, plus 60 B per element-local point
    (ibool, Jacobian, 9 material words) times 25 nspec / nglob."""
    from specfempp_b200 import meshgen, sfg
    steps = args.media_steps
    peak, _ = peaks()
    out = {}
    cases = [("poroelastic_400x400", lambda: meshgen.poroelastic_model(
                  nx=400, nz=400, width=10000.0, height=10000.0, eta_f=1e-3, kxz=2e-10,
                  nstep=2 * steps + 20, layered=True), 112.0, 60.0),
             ("nonconforming_coupled_400_600", lambda: meshgen.nonconforming_coupled(
                  nx_el=400, nx_ac=600, nz_el=200, nz_ac=150, width=40000.0, h_el=20000.0, h_ac=15000.0,
                  nstep=2 * steps + 20), None, None)]
    for name, make, glob_b, loc_b in cases:
        w = make()
        sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=w.nstep)
        sim.set_sources(w.sources)
        sim.set_receivers(w.rec_x, w.rec_z, 0.0, ("displacement",))
        sim.initialize()
        inf = sim.info()
        sim.run(10)
        barrier()
        ms_fl = max_over_ranks(sim.run_timed_flushed(steps))
        ms_b2b = max_over_ranks(sim.run_timed(steps))
        nglob = inf.nglob_elastic + inf.nglob_acoustic
        rec = {"nglob": nglob, "nspec": inf.nspec, "ncomp_elastic": inf.ncomp_elastic,
               "kernel_variant": inf.kernel_variant, "elements_per_block": inf.elements_per_block,
               "steps": steps, "ms_per_step_flushed": ms_fl / steps, "ms_per_step_back_to_back": ms_b2b / steps,
               "gll_pt_updates_per_s": world * nglob * steps / (ms_fl / 1e3),
               "finite": bool(sim.check_finite())}
        if glob_b is not None:
            alg = glob_b + loc_b * 25.0 * inf.nspec / nglob
            rec["algorithmic_bytes_per_point"] = alg
            rec["step_frac_of_hbm"] = alg * nglob / (ms_fl / steps / 1e3) / 1e9 / peak
        out[name] = rec
        sim.close()
    return out


def run_reference(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    w = make_workload(args.workload, max(args.steps, 1))
    # each bench step is one time step of the full model; the timed sample is
    # capped so that warm-up plus timed steps stay near a minute on the host
    steps = max(1, min(args.steps, 3000))
    warm = args.warmup
    cpu_oracle_throughput(w, warm, threads)
    v, secs = cpu_oracle_throughput(w, steps, threads)
    ms = secs * 1000.0 / steps
    nglob = int(round(v * secs / steps))
    cfg = workload_config(args.workload, w, nglob)
    cfg["parallelism"] = "replicas" if args.gpus > 1 else "single GPU"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} time steps of {args.workload} (full mesh), "
                                       f"FP32 C++ restatement of the reference (reference evaluation order), "
                                       f"colour-ordered OpenMP assembly on {threads} threads"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="sfg", choices=["sfg", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-mesh", default="1000x500",
                    help="elements of the batched-shot model, NXxNZ (config 3: 1000x500)")
    ap.add_argument("--batched-shots", type=int, default=32)
    ap.add_argument("--batched-steps", type=int, default=30)
    ap.add_argument("--batched-variant", type=int, default=0,
                    help="assembly of the batched run (1 colour passes, 3 owner-computes, 5 fused tiles; 0 autotuned)")
    ap.add_argument("--kernel-variant", type=int, default=0,
                    help="fix the element-kernel variant of the headline run (0 = autotuned)")
    ap.add_argument("--elements-per-block", type=int, default=0,
                    help="fix the elements per block of the headline run (0 = autotuned)")
    ap.add_argument("--no-3d", action="store_true")
    ap.add_argument("--mesh3d", default="128x128x64")
    ap.add_argument("--steps3d", type=int, default=50)
    ap.add_argument("--epb3d", type=int, default=0,
                    help="3D element kernel launch shape: 1, 2, 4 point form, 6, 8 column form (0 autotuned)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-media", action="store_true")
    ap.add_argument("--media-steps", type=int, default=200)
    ap.add_argument("--adjoint-mesh", default="500x250")
    ap.add_argument("--adjoint-steps", type=int, default=4000)
    ap.add_argument("--adjoint-fd", type=int, default=8,
                    help="finite-difference check along this many perturbations (all 8 sources)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    from specfempp_b200 import sfg
    total_steps = args.warmup + args.steps
    w = make_workload(args.workload, total_steps)
    sim = sfg.Simulation2D(w.mesh, dt=w.dt, nstep=total_steps, kernel_variant=args.kernel_variant,
                           elements_per_block=args.elements_per_block)
    sim.set_sources(w.sources)
    sim.set_receivers(w.rec_x, w.rec_z, types=("displacement",))
    sim.initialize()
    inf = sim.info()
    nglob = inf.nglob

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- value: device-resident, L2 flushed before every timed step ----
    sim.run(args.warmup)
    sim.synchronize()
    clocks = ClockSampler(local)
    barrier()
    ms = sim.run_timed_flushed(args.steps, FLUSH_BYTES)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ms)
    finite = sim.check_finite()
    value = world * nglob * args.steps / (ms / 1000.0)

    # ---- supplementary: back-to-back graph replay (L2 not flushed) ----
    sim.reset()
    sim.run(args.warmup)
    barrier()
    ms_b2b = max_over_ranks(sim.run_timed(args.steps))

    # ---- e2e: per-step C-ABI call with host buffers ----
    sim.reset()
    nsrc = len(w.sources)
    stf_rows = torch.zeros((total_steps, nsrc), dtype=torch.float32).pin_memory().numpy()
    from specfempp_b200 import stf as _stf
    stf_rows[:] = _stf.table(w.sources, w.dt, total_steps)
    seis_row = torch.zeros((inf.nshots, inf.ntypes, inf.nrec, 2), dtype=torch.float32).pin_memory().numpy()
    for i in range(args.warmup):
        sim.step_io(stf_rows[i], seis_row)
    barrier()
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        sim.step_io(stf_rows[i], seis_row)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = world * nglob * args.steps / e2e_s

    # ---- roofline of the dominant kernel ----
    # its launch timed as in the timed region (the L2 flushed before every
    # launch, so every input byte comes from HBM), and back to back
    stiff_ms = sim.time_kernel(0, 50, FLUSH_BYTES)
    stiff_ms_b2b = sim.time_kernel(0, 50)
    upd_ms = sim.time_kernel(1, 50)
    ac_ms = sim.time_kernel(2, 50)
    if inf.kernel_variant >= 3:
        # owner-computes (variants 3, 4, 6; for the fused tile kernel, 5, the
        # element part): the element kernel reads geometry and the gathered field
        # and writes each element point's contribution once (8 B elastic, 4 B acoustic)
        stiff_bytes = ((STIFF_B_PER_LOCAL + 8) * inf.nspec_elastic * 25 + 8 * inf.nglob_elastic +
                       (STIFF_B_PER_LOCAL_AC + 4) * inf.nspec_acoustic * 25 + 4 * inf.nglob_acoustic)
    else:
        stiff_bytes = (STIFF_B_PER_LOCAL * inf.nspec_elastic * 25 + STIFF_B_PER_GLOB * inf.nglob_elastic +
                       STIFF_B_PER_LOCAL_AC * inf.nspec_acoustic * 25 + STIFF_B_PER_GLOB_AC * inf.nglob_acoustic)
    peak, peak_kind = peaks()
    achieved = stiff_bytes / (stiff_ms / 1e3) / 1e9
    tr = traffic_from_profile()
    traffic = None
    if tr and tr.get("workload") == args.workload:
        # the DRAM traffic of the element kernel in use, from its ncu capture
        traffic = tr.get("stiffness_bytes_per_launch_by_variant", {}).get(str(inf.kernel_variant))
    step_bytes = STEP_B_GLOB * nglob + STEP_B_LOCAL * inf.nspec * 25
    kname = ("element kernel, one owner-computes launch of one step" if inf.kernel_variant >= 3 else
             f"element kernel, all {inf.ncolors_elastic} colour launches of one step")
    roofline = {"bound": "hbm", "kernel": f"{kname} (variant {inf.kernel_variant}, "
                                          f"{inf.elements_per_block} elements/block, both media)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": stiff_bytes, "launch_ms": stiff_ms,
                "launch_timing": "CUDA events around each launch, L2 flushed before it (256 MiB written, "
                                 "then another 256 MiB read)",
                "launch_ms_back_to_back": stiff_ms_b2b,
                "frac_back_to_back": stiff_bytes / (stiff_ms_b2b / 1e3) / 1e9 / peak,
                "update_launch_ms": upd_ms, "acoustic_update_launch_ms": ac_ms,
                "step_algorithmic_bytes": step_bytes,
                "step_frac_of_peak": step_bytes / (ms / args.steps / 1e3) / 1e9 / peak}

    batched = None
    if not args.no_batched:
        batched = bench_batched(args, world, barrier, max_over_ranks)

    adj = None
    if not args.no_adjoint:
        adj = bench_adjoint(args, world, barrier, max_over_ranks)

    b3d = None
    if not args.no_3d:
        b3d = bench_3d(args, world, barrier, max_over_ranks)

    media = None
    if not args.no_media:
        media = bench_media(args, world, barrier, max_over_ranks)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        n = sample_steps(20, cpu_oracle_throughput(w, 20, threads)[1], 4000)
        v, secs = cpu_oracle_throughput(w, n, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} time steps of {args.workload} (full mesh), FP32 C++ restatement of the "
                         f"reference on {threads} host threads ({secs:.2f} s)"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    cfg = workload_config(args.workload, w, nglob)
    cfg["parallelism"] = "replicas" if world > 1 else "single GPU"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": cfg,
        "back_to_back": {"value": world * nglob * args.steps / (ms_b2b / 1000.0),
                         "ms_per_step": ms_b2b / args.steps, "l2": "not flushed (graph replay)"},
        "finite": bool(finite),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 4 * nsrc,
                "d2h_bytes_per_step": 4 * inf.nshots * inf.ntypes * inf.nrec * 2},
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": inf.kernels_per_step * args.steps,
        "batched": batched,
        "adjoint": adj,
        "elastic3d": b3d,
        "media": media,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
