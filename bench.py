#!/usr/bin/env python
"""Benchmark: (source, period) forward + adjoint solves/s on one B200.

Workload: the batched configuration -- 301x301 surface grid at 0.01 deg,
400 stations as sources and receivers, 20 periods 2-50 s: 8000 forward +
adjoint solves per step, FP32 sweeps with FP64 T0 / residuals / accumulation,
one persistent launch replayed as a CUDA graph.  Inputs are seeded synthetic
(no public dataset exists for this path).

A step is one misfit evaluation of the whole event set: media preparation,
the fused per-event forward FSM -> receivers -> residuals -> adjoint FSM ->
mask -> FP64 kernel accumulation, and the misfit sum.  Inputs (>= 700 MB of
per-event scratch traffic per step) are larger than L2, so no flush is needed.

`value` is device-timed with CUDA events on the launching stream (max over
ranks); `e2e` times the same step through the public plan API with pinned
host buffers, host->device copies of the step's inputs and the device->host
read of adj_s and the misfit inside the timed region.

--impl reference times the CPU restatement of the reference (oracle/, all
host threads) on a bounded sample of the same workload.
Under torchrun each rank runs its own shard of (source, period) events
(weak scaling); the only exchange is the FP64 all-reduce of adj_s and the
misfit (the reference's MPI_Allreduce, src/preproc.cpp:146, :238).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "(src,period) fwd+adj solves/s, batched FP32 sweeps (FP64 T0/residual/accumulation)"
UNIT = "solves/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--nsta", type=int, default=400)
    p.add_argument("--nper", type=int, default=20)
    p.add_argument("--n", type=int, default=301)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--inversion", type=int, default=0, metavar="K",
                   help="instead of the batch benchmark: K L-BFGS iterations of the full "
                        "inversion loop on the 601x601x50 / 30000-solve workload")
    p.add_argument("--c4", action="store_true",
                   help="instead of the batch benchmark: the uneven topography batch on its "
                        "three grid levels (101, 201, 401), each autotuned")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the misfit-gradient and plain-FP64 side measurements")
    return p.parse_args()


def workload_config(a, world):
    return {"workload": f"C3 batched fwd+adj: {a.n}x{a.n} grid at 0.01 deg, {a.nsta} stations "
                        f"(sources and receivers), {a.nper} periods 2-50 s, "
                        f"{a.nsta * a.nper} events per rank",
            "grid": [a.n, a.n], "stations": a.nsta, "periods": a.nper,
            "events_per_rank": a.nsta * a.nper, "ranks": world,
            "l2_policy": "per-step working set > L2 (126 MB); no flush",
            "phase_velocities": "fwdsurf of the 301x301x40 random-field model (device)",
            "graph": True, "precision": a.precision}


def make_inputs(a, rank, dev=None):
    """The C3 workload and its own Rayleigh phase velocities: SurfGrid::fwdsurf
    of the 3-D random-field model, on the device (sa_surfdisp_columns) or,
    for the CPU reference arm (dev None), by the CPU restatement on every host
    thread -- the two are bit-identical."""
    from surfattpp_b200 import workloads as W
    w = W.config3(seed=1003 + rank, nsta=a.nsta, nper=a.nper, n=a.n)
    if dev is None:
        from oracle import oracle as O
        sv, st = O.fwdsurf(w.zgrid, w.vs3d, w.periods, nthreads=os.cpu_count() or 1)
        return w, sv
    import torch
    from surfattpp_b200 import surfker
    sv, st = surfker.fwdsurf(w.zgrid, torch.as_tensor(np.ascontiguousarray(w.vs3d), device=dev),
                             w.periods)
    torch.cuda.synchronize()
    return w, sv.cpu().numpy()


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, dev):
        self.dev, self.rows, self.stop, self.t = dev, [], False, None

    def __enter__(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self.stop:
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True,
                                         text=True, timeout=5).stdout.strip()
                    if out:
                        self.rows.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                time.sleep(0.2)
        self.t = threading.Thread(target=run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *exc):
        self.stop = True
        self.t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# DRAM bytes moved per algorithmic byte by batch_kernel<float>, from
# dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the same
# kernel on the 151x151 / 3000-event case (45.018 GB moved for 61.719 GB of
# algorithmic bytes; the phase velocities are fwdsurf's of the random-field
# model, as in the full workload).  The algorithmic bytes count every cell of
# every sweep the reference performs; the kernel skips cells that provably
# stay unchanged, so it moves less.  Traffic scales with cell updates, so a
# full launch moves algorithmic x this ratio.
TRAFFIC_PER_ALGO_BYTE = {"fp32": (36.528193e9 + 8.616214e9) / 61.718708e9}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(nx, ny, fwd_iters, adj_iters, bpu_fwd, bpu_adj):
    """Algorithmic HBM bytes of the sweeps: per cell update, each stored
    operand read once and the field written once (forward: T0, T0x, T0y, a,
    b, c, fun, tau + tau write; adjoint: two face fluxes, delta, Ta + Ta
    write), times cell updates = iterations x 4 sweeps x cells."""
    fwd = float(np.sum(fwd_iters)) * 4 * nx * ny
    adj = float(np.sum(adj_iters)) * 4 * (nx - 2) * (ny - 2)
    return fwd * bpu_fwd + adj * bpu_adj, fwd, adj


def cpu_baseline(a, w, svel, nev=None):
    """The oracle (port of the reference) on a bounded sample of events with
    every host thread: 24 events per thread by default (about 10 s on the
    301x301 grid, where one FP64 forward + adjoint solve takes ~0.4 s on one
    core).  Built on this host with the reference's release flags (-O3
    -march=native, GNU C++17)."""
    from oracle import oracle as O
    from surfattpp_b200 import workloads as W
    O.lib("native")
    rng = np.random.default_rng(7)
    nth = os.cpu_count() or 1
    nev = 24 * nth if nev is None else nev
    keep = np.sort(rng.choice(w.n_events, size=min(nev, w.n_events), replace=False))
    sub = W.subset_events(w, keep)
    m11, m12, m22 = sub.media()
    t0 = time.perf_counter()
    O.forward_for_events(sub.xx_deg, sub.yy_deg, svel, m11, m12, m22, sub.events(),
                         calc_adj=True, nthreads=nth, math="native")
    dt = time.perf_counter() - t0
    return {"value": keep.size / dt, "unit": UNIT, "cores": nth, "kind": "port",
            "flags": "-O3 -DNDEBUG -march=native -std=gnu++17 (the reference's release flags)",
            "sample": f"{keep.size} random events of the same workload, fwd+adj, FP64, "
                      f"{dt:.1f} s"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    w, svel = make_inputs(a, 0, None)
    # each step: 8 events per host thread (~3 s), so --steps 5 ends in well
    # under a minute; the sample has no warm-up state
    nev = 8 * (os.cpu_count() or 1)
    base = cpu_baseline(a, w, svel, nev=nev)
    vals = [base["value"]]
    for _ in range(max(a.steps - 1, 0)):
        vals.append(cpu_baseline(a, w, svel, nev=nev)["value"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": nev / v * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": workload_config(a, world),
            "cpu_baseline": {**base, "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _event_ms(stream, fn, steps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def misfit_gradient_timing(a, w, plan, tt, wt, dev, stream):
    """One misfit-gradient evaluation (Inversion::run_forward_adjoint up to
    combine_kernels) on the workload's 3-D model: wall time on the device per
    iteration, plus each stage run alone on the same stream."""
    import torch
    from surfattpp_b200 import inversion, surfker
    cs = stream.cuda_stream
    g = inversion.MisfitGradient(plan, w.zgrid, w.periods)
    vs = torch.as_tensor(np.ascontiguousarray(w.vs3d), device=dev)
    out = g.run(vs, tt, wt, stream=cs)
    for _ in range(2):
        g.run(vs, tt, wt, out=out, stream=cs)
    torch.cuda.synchronize()
    steps = max(1, min(a.steps, 3))
    ms = _event_ms(stream, lambda: g.run(vs, tt, wt, out=out, stream=cs), steps)
    status = int(out["status"][0])
    sv = out["svel"]
    t_disp = _event_ms(stream, lambda: surfker.fwdsurf(w.zgrid, vs, w.periods, stream=cs,
                                                        check=False), steps)
    sen = g.sen(stream=cs)
    # outputs allocated once, outside the timed region
    t_sen = _event_ms(stream, lambda: surfker.depthkernel_hti(w.zgrid, vs, w.periods, sv,
                                                              stream=cs, out=sen), steps)
    t_comb = _event_ms(stream, lambda: surfker.combine_kernels_vs(out["adj_s"], vs, None, *sen,
                                                                 stream=cs), steps)
    o2 = plan.run(sv, tt, wt, stream=cs)
    t_batch = _event_ms(stream, lambda: plan.run(sv, tt, wt, out=o2, stream=cs), steps)
    g.close()
    del sen
    return {"s_per_iter": ms * 1e-3, "unit": "s/iter", "steps": steps, "status": status,
            "model": f"{w.nx}x{w.ny}x{w.nz} vs3d, {w.nper} Rayleigh phase periods, "
                     f"{w.n_events} events",
            "stages_ms_alone": {"fwdsurf": t_disp, "depthkernel": t_sen,
                                "forward_adjoint": t_batch, "combine": t_comb},
            "note": "depth kernels run on a second stream concurrently with the event batch"}


def pde_smooth_timing(a, w, dev, stream, peak):
    """PostProc::pde_smooth of a kernel on the workload's 3-D grid: device time
    per Euler step and HBM throughput (16 B algorithmic per cell per step: one
    read, one write)."""
    import torch
    from surfattpp_b200 import postproc
    from surfattpp_b200 import workloads as W
    cs = stream.cuda_stream
    # the largest model grid (601 x 601 x 50 at 0.005 deg, 2 km): 144 MB > L2
    xx, yy = W._grid(102.0, 24.0, (601, 601), 0.005)
    zg = np.arange(0.0, 98.0 + 1e-9, 2.0)
    w = type("G", (), dict(nx=601, ny=601, nz=zg.size, xx_deg=xx, yy_deg=yy, zgrid=zg))
    shape = (w.nx, w.ny, w.nz)
    g = torch.Generator(device=dev).manual_seed(11)
    f = torch.rand(shape, dtype=torch.float64, device=dev, generator=g)
    work = torch.empty_like(f)
    d = float(w.xx_deg[1] - w.xx_deg[0])
    dz = float(w.zgrid[1] - w.zgrid[0])
    sig = (5.0 * d, 3.0 * dz)
    postproc.pde_smooth(f, w.yy_deg, w.zgrid, d, d, dz, *sig, work=work, stream=cs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _, ns = postproc.pde_smooth(f, w.yy_deg, w.zgrid, d, d, dz, *sig, work=work, stream=cs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    per = ms / ns
    gbs = 16.0 * f.numel() / (per * 1e-3) / 1e9
    return {"grid": list(shape), "sigma": [sig[0], sig[1]], "nstep": ns, "ms_total": ms,
            "ms_per_step": per, "achieved_gbs": gbs, "frac_of_hbm": gbs / peak,
            "note": "per step one read and one write of the field (16 B per cell); "
                    "field %.0f MB" % (f.numel() * 8 / 1e6)}


def topo_media_timing(dev, stream):
    """SurfGrid::build_media_matrix_with_topo on the 201 x 201 topography
    level: gridding, then per period the geographic Gaussian smoothing,
    gradient, dip angle and media (15 periods)."""
    import torch
    from surfattpp_b200 import surfgrid
    from surfattpp_b200 import workloads as W
    w = W.config4(level=201, nsta=41, src_range=(3, 5), lam=4.0)
    lon, lat, z = w.meta["topo_raw"]
    avg = surfgrid.average_phase_velocity(w.zgrid, w.meta["vs1d"], w.periods)
    sig = surfgrid.sigma_deg(avg, w.periods, w.meta["wavelen_factor"])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    zg = surfgrid.grid_topography(lon, lat, z, w.xx_deg, w.yy_deg)
    surfgrid.build_media_with_topo(w.xx_deg, w.yy_deg, zg, sig, stream=stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return {"grid": [w.nx, w.ny], "periods": int(w.nper), "sigma_deg_range": [float(sig.min()),
            float(sig.max())], "ms_total": e0.elapsed_time(e1)}


def fp64_timing(a, w, sv, tt, wt, dev, stream, ctx, timed=True):
    """The same solves with the FP64 parity path (the reference's arithmetic).
    Also returns its per-event sweep iteration counts, which are the oracle's
    (the FP64 parity tests assert equality): the roofline's algorithmic work
    is counted with them."""
    import torch
    from surfattpp_b200 import preproc
    cs = stream.cuda_stream
    ev = w.events()
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64", ctx=ctx, graph=True)
    out = plan.run(sv, tt, wt, stream=cs)
    torch.cuda.synchronize()
    fi = out["fwd_iters"].cpu().numpy()[:w.n_events].copy()
    ai = out["adj_iters"].cpu().numpy()[:w.n_events].copy()
    res = None
    if timed:
        plan.run(sv, tt, wt, out=out, stream=cs)
        torch.cuda.synchronize()
        steps = max(1, min(a.steps, 2))
        ms = _event_ms(stream, lambda: plan.run(sv, tt, wt, out=out, stream=cs), steps)
        res = {"value": w.n_events / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
               "steps": steps, "dtype": "f64"}
    plan.close()
    return res, fi, ai


def exact_gradient_timing(a, w, tt, wt, dev, stream, ctx):
    """The exact gradient of the discrete forward model on the same
    workload: an FP64 plan with the discrete adjoint (forward solves to a
    fixed point), fwdsurf and the phase-velocity root derivatives, one fused
    evaluation (sa_grad_run) per step."""
    import torch
    from surfattpp_b200 import inversion, preproc
    cs = stream.cuda_stream
    ev = w.events()
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp64", ctx=ctx, graph=True)
    plan.set_adjoint("exact")
    g = inversion.MisfitGradient(plan, w.zgrid, w.periods)
    vs = torch.as_tensor(np.ascontiguousarray(w.vs3d), device=dev)
    out = g.run(vs, tt, wt, stream=cs)
    g.run(vs, tt, wt, out=out, stream=cs)
    torch.cuda.synchronize()
    steps = max(1, min(a.steps, 2))
    ms = _event_ms(stream, lambda: g.run(vs, tt, wt, out=out, stream=cs), steps)
    status = int(out["status"][0])
    g.close()
    plan.close()
    return {"s_per_iter": ms * 1e-3, "unit": "s/iter", "steps": steps, "status": status,
            "dtype": "f64",
            "note": "fwdsurf, every forward solve to a fixed point, the exact discrete "
                    "adjoint, dc/dvs from the phase-velocity roots, combination"}


def per_solve_timing(w, svel, nev=4):
    """The plain per-solve form: FP64, one forward and one adjoint call per
    event through the single-solve C ABI with host arrays, as the reference's
    forward_for_event calls eikonal::FSM_UW_PS_lonlat_2d and
    FSM_O1_JSE_lonlat_2d (src/preproc.cpp:88-127), receiver interpolation and
    residuals on the host."""
    from surfattpp_b200 import eikonal
    m11, m12, m22 = w.media()
    ev = w.events()
    X, Y = w.xx_deg, w.yy_deg
    dx, dy = X[1] - X[0], Y[1] - Y[0]

    def bilinear(T, x, y):
        i = np.clip(((x - X[0]) / dx).astype(int), 0, X.size - 2)
        j = np.clip(((y - Y[0]) / dy).astype(int), 0, Y.size - 2)
        r, q = (x - X[i]) / dx, (y - Y[j]) / dy
        return ((1 - r) * (1 - q) * T[j, i] + r * (1 - q) * T[j, i + 1]
                + (1 - r) * q * T[j + 1, i] + r * q * T[j + 1, i + 1])

    rng = np.random.default_rng(11)
    keep = np.sort(rng.choice(w.n_events, size=min(nev + 1, w.n_events), replace=False))
    t0 = time.perf_counter()
    for i, e in enumerate(keep):
        if i == 1:               # the first solve warms the path up, untimed
            t0 = time.perf_counter()
        ip = int(ev["iper"][e])
        a0, b0, c0 = m11[ip], m22[ip], -m12[ip]
        T = eikonal.FSM_UW_PS_lonlat_2d(X, Y, a0, b0, c0, 1.0 / svel[ip], ev["evlo"][e],
                                        ev["evla"][e])
        r = ev["rec_idx"][ev["rec_ptr"][e]:ev["rec_ptr"][e + 1]]
        o = slice(ev["rec_ptr"][e], ev["rec_ptr"][e + 1])
        xr, yr = ev["stlo"][r], ev["stla"][r]
        sadj = ev["weight"][o] * (bilinear(T, xr, yr) - ev["tt_obs"][o])
        Ta = eikonal.FSM_O1_JSE_lonlat_2d(X, Y, a0, b0, c0, T, xr, yr, sadj)
        eikonal.mask_uniform_grid(X, Y, Ta, ev["evlo"][e], ev["evla"][e])
    dt = time.perf_counter() - t0
    n = max(keep.size - 1, 1)
    return {"value": n / dt, "unit": UNIT, "events": int(n), "dtype": "f64",
            "note": "one FP64 forward + adjoint solve per call (single-solve C ABI, host "
                    "arrays, wall clock)"}


def run_inversion(a):
    """The full inversion loop on the device (Inversion::run_inversion,
    src/inversion.cpp:106-160): misfit gradient with FP32 sweeps (through the
    torch.autograd.Function backward; forward fields recomputed per event,
    never stored), PDE kernel
    smoothing, FP64 L-BFGS with the strong-Wolfe line search, multiplicative
    model update.  Observed times are the engine's FP32 synthetic times in the
    GRF model; the inversion starts from the 1-D gradient.  Reports wall time
    per L-BFGS iteration and per misfit-gradient evaluation (synchronised)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    print(json.dumps(inversion_timing(a.inversion, dev)), flush=True)
    return 0


def inversion_timing(niter, dev):
    """run_inversion's measurement: `niter` L-BFGS iterations on C5."""
    import torch
    from surfattpp_b200 import inversion, preproc, surfker
    from surfattpp_b200 import workloads as W
    w = W.config5()
    ev = w.events()
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=dev)
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision="fp32", graph=True)
    g = inversion.MisfitGradient(plan, w.zgrid, w.periods)
    wt = t(ev["weight"])
    sv, st = surfker.fwdsurf(w.zgrid, t(w.vs3d), w.periods)
    o = plan.run(sv, t(ev["tt_obs"]), wt, calc_adj=False)
    torch.cuda.synchronize()
    tt_obs = o["syn"][: w.rec_idx.size].clone()
    del o, sv
    smooth = dict(ygrid=w.yy_deg, zgrid=w.zgrid, dx=0.005, dy=0.005, dz=2.0, sigma_h=0.025,
                  sigma_v=6.0)
    # the gradient taken through the fused torch.autograd.Function (one
    # forward-residual-adjoint pass per evaluation, as run_forward_adjoint)
    inv = inversion.Inversion(g, tt_obs, wt, smooth=smooth, niter=niter, autograd="fused")
    vs0 = t(w.meta["vs_start"])
    inv.run_forward_adjoint(vs0)          # graph capture and first-touch, untimed
    count = [0]
    orig = inv.run_forward_adjoint

    def counted(vs):
        count[0] += 1
        return orig(vs)

    inv.run_forward_adjoint = counted
    inv.misfit = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    inv.run(vs0)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    n_it = len(inv.misfit)
    # one gradient through TravelTimes (vs -> receiver times; the backward
    # recomputes every forward field and drives the adjoint with w (T - Tobs))
    v = vs0.detach().clone().requires_grad_(True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    inversion.misfit(g, v, tt_obs, wt).backward()
    torch.cuda.synchronize()
    t_tt = time.perf_counter() - t1
    line = {"metric": "full inversion loop: wall time per L-BFGS iteration", "impl": "b200",
            "value": dt / n_it, "unit": "s/iter", "n_gpus": 1, "steps": n_it,
            "higher_is_better": False, "dtype": "f32",
            "data": "synthetic (seeded GRF model, observed = engine synthetic times)",
            "config": {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "stations": int(w.stlo.size),
                       "periods": int(w.nper), "solves_per_gradient": int(w.n_events),
                       "smoothing_sigma": [0.025, 6.0]},
            "gradient_evaluations": count[0],
            "s_per_gradient": dt / max(count[0], 1),
            "s_per_gradient_travel_times": t_tt,
            "misfit": [float(m) for m in inv.misfit], "alphas": inv.alphas,
            "sub_iters": inv.sub_iters, "restarts": inv.restarts, "wall_s": dt}
    g.close()
    plan.close()
    return line


def c4_levels(dev):
    """The uneven batch with topography: per grid level (101^2, 201^2, 401^2
    over one span) the fractal-topography media (SurfGrid::
    build_media_matrix_with_topo on the device), 15 periods with U{50..600}
    sources and Poisson(40) receivers each, FP32 sweeps on the general-metric
    path.  Each level's launch configuration is autotuned on its own events,
    then three evaluations are timed around the batch kernel.  Then all
    levels' events in ONE persistent launch (sa_multi: per-event grid,
    queue ordered by work across levels, the 401^2 level's tuned variant),
    warmed up once and timed over three evaluations."""
    import torch
    from surfattpp_b200 import preproc, surfgrid
    from surfattpp_b200 import workloads as W
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=dev)
    levels, keep = [], []
    for level in (101, 201, 401):
        w = W.config4(level=level)
        ev = w.events()
        lon, lat, z = w.meta["topo_raw"]
        avg = surfgrid.average_phase_velocity(w.zgrid, w.meta["vs1d"], w.periods)
        sig = surfgrid.sigma_deg(avg, w.periods, w.meta["wavelen_factor"])
        zg = surfgrid.grid_topography(lon, lat, z, w.xx_deg, w.yy_deg)
        m11, m12, m22, _ = surfgrid.build_media_with_topo(w.xx_deg, w.yy_deg, zg, sig)
        X, Y = np.meshgrid(w.xx_deg, w.yy_deg)
        svel = np.stack([avg[k] * (1.0 + 0.03 * np.sin(9 * X + k) * np.cos(7 * Y))
                         for k in range(w.nper)])
        plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                          ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                          ev["stla"], precision="fp32")
        sv, tt, wt = t(svel), t(ev["tt_obs"]), t(ev["weight"])
        out = plan.run(sv, tt, wt, m11=m11, m12=m12, m22=m22)
        tune = plan.autotune(sv, tt, wt, m11=m11, m12=m12, m22=m22, adj_s=out["adj_s"])
        plan.kernel_timing(True)
        ms = []
        for _ in range(3):
            plan.run(sv, tt, wt, m11=m11, m12=m12, m22=m22, out=out)
            ms.append(plan.kernel_ms())
        torch.cuda.synchronize()
        ms = float(np.median(ms))
        levels.append({"grid": [w.nx, w.ny], "events": int(w.n_events),
                       "observations": int(w.rec_idx.size), "kernel_ms": ms,
                       "solves_per_s": w.n_events / (ms * 1e-3),
                       "status": int(out["status"][: w.n_events].max()),
                       "tuned": {k: tune[k] for k in ("choice", "variant", "active_slots")},
                       "candidates_ms": [round(x, 3) for x in tune["ms"]]})
        keep.append((plan, sv, tt, wt, (m11, m12, m22), w.n_events))
    # one launch over the three levels, finest first (its variant applies)
    keep = keep[::-1]
    multi = preproc.MultiPlan([k[0] for k in keep])
    args = [[k[i] for k in keep] for i in (1, 2, 3)]
    media = [[k[4][j] for k in keep] for j in range(3)]
    outs = multi.run(*args, m11=media[0], m12=media[1], m22=media[2])
    ms = []
    for _ in range(3):
        multi.run(*args, m11=media[0], m12=media[1], m22=media[2], outs=outs)
        ms.append(multi.kernel_ms())
    torch.cuda.synchronize()
    ms = float(np.median(ms))
    nev = sum(k[5] for k in keep)
    one = {"kernel_ms": ms, "events": nev, "solves_per_s": nev / (ms * 1e-3),
           "status": multi.worst_status(),
           "sum_of_levels_ms": sum(l["kernel_ms"] for l in levels)}
    multi.close()
    for k in keep:
        k[0].close()
    return levels, one


def run_c4(a):
    import torch
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    levels, one = c4_levels(dev)
    tot_ev = sum(l["events"] for l in levels)
    tot_ms = one["kernel_ms"]
    line = {"metric": "(src,period) fwd+adj solves/s, uneven topography batch (three grid levels)",
            "impl": "b200", "value": tot_ev / (tot_ms * 1e-3), "unit": "solves/s", "n_gpus": 1,
            "steps": 3, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded fractal topography, Poisson receivers)",
            "config": {"workload": "C4 uneven batch with topography, levels 101/201/401, "
                                   "15 periods, U{50..600} sources per period"},
            "levels": levels, "one_launch": one}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.inversion > 0:
        return run_inversion(a)
    if a.c4:
        return run_c4(a)
    import torch
    from surfattpp_b200 import distributed, preproc
    from surfattpp_b200._capi import Context

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    ctx = Context(local)
    w, svel = make_inputs(a, rank, dev)
    ev = w.events()
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    cs = stream.cuda_stream
    plan = preproc.ForwardAdjointPlan(w.xx_deg, w.yy_deg, w.nper, ev["evlo"], ev["evla"],
                                      ev["iper"], ev["rec_ptr"], ev["rec_idx"], ev["stlo"],
                                      ev["stla"], precision=a.precision, ctx=ctx, graph=True)
    t = lambda x: torch.as_tensor(np.ascontiguousarray(x), device=dev)
    sv, tt, wt = t(svel), t(ev["tt_obs"]), t(ev["weight"])
    out = plan.run(sv, tt, wt, stream=cs)

    def step():
        plan.run(sv, tt, wt, out=out, stream=cs)
        if dist is not None:
            distributed.reduce_gradient(out["adj_s"], out["chi"])

    for _ in range(max(a.warmup, 3)):
        step()
    torch.cuda.synchronize()
    fwd_iters = out["fwd_iters"].cpu().numpy()[:w.n_events]
    adj_iters = out["adj_iters"].cpu().numpy()[:w.n_events]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    if dist is not None:
        m = torch.tensor([ms], device=dev)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        ms = float(m)
        dist.barrier()
    status = int(out["status"][:w.n_events].max())

    # the dominant kernel alone: CUDA events around each batch launch (same
    # stream, launched without the graph), one step at a time
    plan.kernel_timing(True)
    kms = []
    for _ in range(a.steps):
        step()
        kms.append(plan.kernel_ms())
    plan.kernel_timing(False)
    torch.cuda.synchronize()
    kernel_ms = float(np.mean(kms))

    # end to end through the public API: pinned host inputs in, adj_s + misfit out
    h_sv = torch.from_numpy(svel).pin_memory()
    h_tt = torch.from_numpy(np.ascontiguousarray(ev["tt_obs"])).pin_memory()
    h_wt = torch.from_numpy(np.ascontiguousarray(ev["weight"])).pin_memory()
    h_adj = torch.empty(out["adj_s"].shape, dtype=torch.float64).pin_memory()
    h_chi = torch.empty(1, dtype=torch.float64).pin_memory()

    def e2e_step():
        sv.copy_(h_sv, non_blocking=True)
        tt.copy_(h_tt, non_blocking=True)
        wt.copy_(h_wt, non_blocking=True)
        step()
        h_adj.copy_(out["adj_s"], non_blocking=True)
        h_chi.copy_(out["chi"], non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(a.steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1) / a.steps
    if dist is not None:
        m = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        ms_e2e = float(m)
    h2d = h_sv.numel() * 8 + h_tt.numel() * 8 + h_wt.numel() * 8
    d2h = h_adj.numel() * 8 + 8

    extra = {}
    timed64 = world == 1 and not a.no_extras
    fp64, fi64, ai64 = fp64_timing(a, w, sv, tt, wt, dev, stream, ctx, timed=timed64)
    if timed64:
        extra["misfit_gradient"] = misfit_gradient_timing(a, w, plan, tt, wt, dev, stream)
        extra["exact_gradient"] = exact_gradient_timing(a, w, tt, wt, dev, stream, ctx)
        extra["fp64_plain"] = fp64
        extra["fp64_per_solve"] = per_solve_timing(w, svel)
        extra["pde_smooth"] = pde_smooth_timing(a, w, dev, stream, peaks()[0])
        extra["topo_media"] = topo_media_timing(dev, stream)

    if rank == 0:
        peak, peak_kind = peaks()
        bpu_f, bpu_a = (36, 20) if a.precision == "fp32" else (72, 40)
        # work counted with the FP64 (oracle) iteration counts per event
        algo, nf, na = algorithmic_bytes(w.nx, w.ny, fi64, ai64, bpu_f, bpu_a)
        achieved = algo / (kernel_ms * 1e-3) / 1e9
        total_events = w.n_events * world
        line = {
            "metric": METRIC, "value": total_events / (ms * 1e-3), "unit": UNIT,
            "n_gpus": world, "steps": a.steps, "warmup": max(a.warmup, 3),
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if a.precision == "fp32" else "f64",
            "data": "synthetic (seeded GRF model, straight-ray observed times)",
            "config": workload_config(a, world),
            "e2e": {"value": total_events / (ms_e2e * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            # per step: media64, [media32], batch, sum_events, fold_status,
            # event_cost (the queue-order sort is CUB, not counted)
            "gpu_launches": (6 if a.precision == "fp32" else 5) * a.steps,
            "cell_updates_per_s": (nf + na) / (ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (algo * TRAFFIC_PER_ALGO_BYTE[a.precision]
                                     if a.precision in TRAFFIC_PER_ALGO_BYTE else None),
                         "traffic_source": "ncu dram bytes of the 151x151 capture, scaled "
                                           "by cell updates",
                         "kernel": "batch_kernel<%s>" % ("float" if a.precision == "fp32"
                                                         else "double"),
                         "kernel_ms": kernel_ms, "algorithmic_bytes": algo,
                         "peak_kind": peak_kind,
                         "note": "algorithmic bytes: 36 B per forward / 20 B per adjoint "
                                 "cell update (FP32), x2 for FP64, over iterations x 4 sweeps "
                                 "x cells with the FP64 plan's (= the oracle's) per-event "
                                 "iteration counts",
                         "iterations": {"fp64_fwd": int(fi64.sum()), "fp64_adj": int(ai64.sum()),
                                        "run_fwd": int(fwd_iters.sum()),
                                        "run_adj": int(adj_iters.sum())}},
            "clocks": clk.summary(),
            "status": status,
        }
        line.update(extra)
    plan.close()
    if rank == 0:
        if timed64:
            # the other two measured configurations, so that one default run
            # reports them: the uneven topography batch (per level) and the
            # full inversion loop on 601x601 (two L-BFGS iterations)
            import gc
            gc.collect()
            torch.cuda.empty_cache()
            lv, one = c4_levels(dev)
            line["c4_uneven_topography"] = {"solves_per_s": one["solves_per_s"],
                                            "one_launch": one, "levels": lv}
            gc.collect()
            torch.cuda.empty_cache()
            inv = inversion_timing(2, dev)
            line["c5_inversion"] = {k: inv[k] for k in ("value", "unit", "config",
                                                        "s_per_gradient", "gradient_evaluations",
                                                        "s_per_gradient_travel_times",
                                                        "misfit", "alphas", "wall_s")}
        if not a.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(a, w, svel)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
