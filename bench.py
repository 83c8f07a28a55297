#!/usr/bin/env python3
"""Benchmark: ray-surfaces/s of the cross-dispersed echelle (1e8 rays) on B200.

Workload (one step): the C1 scheme -- off-axis parabola, echelle (orders
30..60, one beam per order), cross-disperser, toric fold, two-surface
even-asphere lens, CCD 4096^2 -- traced for 31 x 64 x 50,404 = 1.0e8 rays
resident in HBM (5.7 GB of input, far larger than the 126 MB L2), with the
CCD frame counts accumulated.  A ray-surface is one ray through one non-Aux
surface; lost rays count up to the surface that loses them.

Engines timed: the plain FP64 per-surface engine (one kernel per surface,
rtb_trace_out), the fused FP64 kernel and the two fused mixed-precision
kernels (FP64 ray state, RTB_MIXED; FP32 ray state, RTB_MIXED32), each fused
kernel as a plan (rtb_plan_*: rays resident in HBM as 32-ray row blocks in a
coherent tracing order, outputs stored at the tracing slots, one CUDA graph
launch per step, launch configuration chosen by the autotuner first).  The
headline `value` is the faster mixed kernel whose p99.9 CCD error against
the FP64 plan is within 0.05 um.  `e2e` runs the same trace through rtb_trace_host on
page-locked host arrays (copies in and out inside the timed region).
`cpu_baseline` is the CPU oracle on the host cores over a bounded sample of
the same rays.  `c3_batched` is C3: 512 beams of uneven size, wavelength,
field angle and order through the same scheme in one graph launch.
`c4_adjoint` is C4: the forward/backward pair that gives the gradient of
the spot merit in 24 scheme parameters over 1e7 rays.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from rt_b200.clocks import Clocks  # noqa: E402

METRIC = "ray·surfaces/s on 1 B200, fused mixed vs plain FP64 at ≤0.05µm CCD error"
UNIT = "ray·surfaces/s"
WORKLOAD = ("C1 cross-dispersed echelle: 1.0e8 rays (31 echelle orders 30..60 x 64 wavelengths 0.38-0.90 um "
            "x 50404 rays, disk r=25 mm), OAP + echelle + cross-disperser + toric fold + 2 even-asphere lens "
            "surfaces + CCD 4096^2, frame counts accumulated")
FIXES = 3  # RTB_FIX_TORIC_SIGN | RTB_FIX_TORIC_STEP: the toric fold's Steffensen step divides 0/0 otherwise
# Per-ray figures of the two mixed kernels (compiled for C1 with its surface
# constants baked in; plans with slot outputs), from ncu captures of one
# launch each: DRAM bytes read + written on this workload (1.0e8 rays, one
# pass), and the executed FP64 / FP32 floating-point operations on C1 at
# 1.0e7 rays (31 x 64 x 5041; ncu op counters, FMA = 2, FFMA2 = 4).
KERNEL_PROFILE = {
    "fused_mixed": {"traffic_per_ray": 76.92, "f64_flops_per_ray": 526.64, "f32_flops_per_ray": 52.17},
    "fused_mixed32": {"traffic_per_ray": 52.06, "f64_flops_per_ray": 385.37, "f32_flops_per_ray": 237.10},
}
# bytes of input per ray the mixed kernels read: a plan's 32-ray row blocks
# (Row64: 1824 B, Row32: 1056 B per 32 rays)
ROW_BYTES_PER_RAY = {"fused_mixed": 1824 / 32, "fused_mixed32": 1056 / 32}
# bytes per ray-surface of a minimal per-surface FP64 pass: read X..cZ, lambda,
# flag (57 B), write X..cZ, flag (49 B)
ALG_BYTES_PER_RAY_SURFACE = 106


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--rays-per-lambda", type=int, default=0, help="override (default: 1e8 rays total)")
    p.add_argument("--surfaces", type=int, default=0,
                   help="profiling: trace only the scheme's first K surfaces (per-surface cost by difference)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-c3", action="store_true")
    p.add_argument("--no-c4", action="store_true")
    p.add_argument("--c4-rays-per-lambda", type=int, default=156250, help="C4 adjoint: rays per wavelength (x64)")
    p.add_argument("--no-autotune", action="store_true", help="default launch configuration (profiling runs)")
    p.add_argument("--engines", default="per_surface,fused_fp64,fused_mixed,fused_mixed32")
    return p.parse_args()


def dist_init(args):
    from rt_b200 import replicas
    return replicas.init("nccl")


def cpu_baseline(specs_fn, beams_all, budget_s=12.0, runs=5):
    """CPU oracle on all host threads over a bounded sample: the first m rays
    of every beam, m sized so that `runs` timed runs take ~budget_s seconds;
    the rate is that of the median run (after one warm-up run)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    from rt_b200 import schemes as S
    lib = O.load()
    threads = lib.oracle_num_threads()
    cs = S.to_c(specs_fn(), O.spline_init)

    def run(m):
        beams, first = [], 0
        for b in beams_all:
            nb = S.make_beam(first, 1, 1, 1.0, (0.5, 0.5), 0)
            nb.first_ray, nb.n_rays = first, min(m, int(b.n_rays))
            for i in range(b.n_orders):
                nb.orders[i] = b.orders[i]
            nb.n_orders = b.n_orders
            nb.disk[:] = b.disk[:]
            nb.range[:] = b.range[:]
            nb.n_lambda = b.n_lambda
            nb.seed = b.seed
            beams.append(nb)
            first += nb.n_rays
        rays = O.generate(beams, first)
        t0 = time.perf_counter()
        st, stats, _ = O.trace(cs.surfaces, beams, rays, fixes=FIXES)
        dt = time.perf_counter() - t0
        return first, stats.ray_surfaces, dt

    n, rs, dt = run(2000)
    rate = rs / dt
    m = int(min(max(2000, budget_s / runs * rate / (len(beams_all) * 5.3)), int(beams_all[0].n_rays)))
    run(m)  # warm-up
    timed = sorted((run(m) for _ in range(runs)), key=lambda r: r[2])
    n, rs, dt = timed[len(timed) // 2]
    # one core on a smaller sample, for the per-core figure
    lib.oracle_set_threads(1)
    m1 = max(200, m // max(1, threads))
    n1, rs1, dt1 = run(m1)
    lib.oracle_set_threads(threads)
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            model = next((ln.split(":", 1)[1].strip() for ln in f if ln.startswith("model name")), "")
    except OSError:
        pass
    return {"value": rs / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"first {m} rays of each of the {len(beams_all)} order beams ({n} rays, {rs} ray-surfaces), "
                      f"CPU oracle (C++, OpenMP, FP64), median of {runs} runs after a warm-up: {dt:.2f} s",
            "one_core": {"value": rs1 / dt1, "sample": f"first {m1} rays of each beam ({n1} rays), {dt1:.2f} s"},
            "nproc": os.cpu_count(), "cpu_model": model}


def c4_adjoint(npl, reps=3):
    """C4: the adjoint pair on the C0 spectrograph with its asphere field
    flattener, 64 wavelengths x npl rays, 24 parameters.  The merit
    sum_lambda RMS_spot + 10 (x_mean - x_t(lambda))^2 and its per-ray seeds
    come from rtb_adjoint_spot_merit; one forward with checkpoints, the merit
    and one backward give its whole gradient; likewise the spectral-resolution
    merit (rtb_adjoint_resolution_merit).  Each call returns
    synchronised: wall-clock times, best of reps."""
    import torch
    from rt_b200 import engine as E
    from rt_b200 import ffi, schemes as S
    cs = S.to_c(S.littrow_free_asphere(), E.spline_init)
    beams = S.c4_beams(n_per_lambda=npl)
    n = S.total_rays(beams)
    rays = E.generate(beams, n)
    torch.cuda.synchronize()
    adj = E.Adjoint(cs.surfaces, S.c4_params(), beams, n, fixes=ffi.FIX_ASPHERE_ROOT)
    theta = adj.theta()
    lam = np.linspace(S.C4_LAMBDA[0], S.C4_LAMBDA[1], S.C4_NLAMBDA)
    target = S.c4_target_x(lam)

    def best(fn):
        out, ts = None, []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return min(ts) * 1e3, out

    t_fwd, (st, stats) = best(lambda: adj.forward(theta, rays))
    ffi.check(st, "rtb_adjoint_forward")
    t_mer, (merit, gX, gY) = best(lambda: adj.spot_merit(target, 10.0))
    t_bwd, grad = best(lambda: adj.backward(gX, gY))
    d = np.zeros(len(theta))
    d[0] = 1.0
    t_jvp, _ = best(lambda: adj.jvp(d))
    # the spectral-resolution merit (sum of inverse resolving powers along x)
    # and its gradient by the same backward
    t_res, (res_merit, rX, rY) = best(lambda: adj.resolution_merit(lam))
    t_rbwd, rgrad = best(lambda: adj.backward(rX, rY))
    P = len(theta)
    res = {"n_rays": n, "n_good": stats.n_good, "n_params": P, "merit": merit,
           "forward_ms": t_fwd, "merit_ms": t_mer, "backward_ms": t_bwd, "jvp_ms_per_direction": t_jvp,
           "gradient_ms": t_fwd + t_mer + t_bwd, "central_differences_ms": 2 * P * t_fwd,
           "grad_norm": float(np.linalg.norm(grad)),
           "resolution_merit": {"merit": res_merit, "merit_ms": t_res, "gradient_ms": t_fwd + t_res + t_rbwd,
                                "grad_norm": float(np.linalg.norm(rgrad))},
           "how": "rtb_adjoint_forward (checkpoints at surface inputs), rtb_adjoint_spot_merit, "
                  "rtb_adjoint_backward (reverse sweep inside each surface, compiled for the scheme's structure), rtb_adjoint_jvp; "
                  "wall clock of synchronous calls, best of 3"}
    adj.destroy()
    del rays
    torch.cuda.empty_cache()
    return res


def dgemm_tflops(n=4096, reps=5):
    """cuBLAS FP64 GEMM throughput on this GPU (TFLOP/s, best of reps)."""
    import torch
    try:
        a = torch.randn(n, n, dtype=torch.float64, device="cuda")
        b = torch.randn(n, n, dtype=torch.float64, device="cuda")
        torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    except RuntimeError:
        return None


def sgemm_tflops(n=8192, reps=5):
    """cuBLAS FP32 GEMM throughput with TF32 off (the FP32 pipes), TFLOP/s."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    try:
        torch.backends.cuda.matmul.allow_tf32 = False
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        torch.matmul(a, b)
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    except RuntimeError:
        return None
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def workload_config(n_rays, n_beams):
    """The `config` of both arms' lines: the workload, not the engine."""
    return {"workload": WORKLOAD, "n_rays": n_rays, "beams": n_beams, "l2": "inputs (3.3-5.7 GB) larger than L2",
            "toric_fixes": FIXES}


def reference_arm(args):
    # rank 0 alone runs (on the host cores) and prints; the other ranks exit
    from rt_b200 import replicas
    world, rank, _ = replicas.env()
    if rank != 0:
        return
    from rt_b200 import schemes as S
    beams = S.c1_beams()
    res = cpu_baseline(S.echelle, beams, budget_s=min(30.0, max(2.0, 0.3 * args.steps)))
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(S.total_rays(beams), len(beams)),
            "engine": "CPU oracle (restatement of cuda_engine math; the reference's CPU engine simd_engine is a "
                      "non-functional stub), on a bounded sample of the workload (cpu_baseline.sample)",
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    world, rank, local = dist_init(args)
    torch.cuda.set_device(local)
    from rt_b200 import engine as E
    from rt_b200 import ffi, schemes as S

    npl = args.rays_per_lambda or S.c1_rays_per_lambda()
    from rt_b200 import replicas
    beams = S.c1_beams(n_per_lambda=npl, seed=replicas.seed(S.SEED, rank))
    n = S.total_rays(beams)
    specs = S.echelle()
    if args.surfaces > 0:
        specs = specs[:args.surfaces]
    cs = S.to_c(specs, E.spline_init)
    surf = cs.surfaces
    rays_in = E.generate(beams, n)
    torch.cuda.synchronize()  # generated on the library's stream
    out = E.DeviceRays(n)
    ccd = S.ccd(S.C1_CCD)
    counts = torch.zeros(int(ccd.xdim) * int(ccd.ydim), dtype=torch.int32, device="cuda")
    outside = torch.zeros(1, dtype=torch.int64, device="cuda")
    import ctypes as C
    L = E.lib()
    L.rtb_trace_out.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                                C.POINTER(ffi.TraceOpts), C.POINTER(ffi.Rays), C.POINTER(ffi.Rays),
                                C.POINTER(ffi.TraceStats), C.c_void_p]
    s_arr = (ffi.Surface * len(surf))(*surf)
    b_arr = (ffi.Beam * len(beams))(*beams)
    rin, rout = rays_in.struct(), out.struct()
    # a stream of its own: a NULL handle (torch's default stream) would send
    # the library's work to the library's own stream, outside the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def step(o):
        stats = ffi.TraceStats()
        st = L.rtb_trace_out(s_arr, len(surf), b_arr, len(beams), C.byref(o), C.byref(rin), C.byref(rout),
                             C.byref(stats), C.c_void_p(stream.cuda_stream))
        ffi.check(st, "rtb_trace_out")
        return stats

    # device time of K steps, the maximum over ranks; `rs` the ray-surfaces of
    # one step summed over ranks (each replica traces its own rays)
    def timed(o, K, W):
        for _ in range(W):
            stats = step(o)
        replicas.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            stats = step(o)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = replicas.max_over_ranks(e0.elapsed_time(e1))
        stats.rs = replicas.sum_over_ranks(stats.ray_surfaces)
        return ms / K, stats

    engines = {}
    mk = lambda eng, prec, out_order=ffi.OUT_INDEX: E.opts(engine=eng, precision=prec, fixes=FIXES, state_out=0,  # noqa
                                                          ccd=ccd, counts=counts, n_outside=outside,
                                                          out_order=out_order)
    FUSED = (("fused_fp64", ffi.FP64), ("fused_mixed", ffi.MIXED), ("fused_mixed32", ffi.MIXED32))
    MIXED_ENGINES = {"fused_mixed": ffi.MIXED, "fused_mixed32": ffi.MIXED32}
    PREC = dict(FUSED)
    KERNELS = {ffi.FP64: ("rtb_fused_fp64_scheme", "k_fused_fp64"),
               ffi.MIXED: ("rtb_fused_mixed_scheme", "k_fused_mixed"),
               ffi.MIXED32: ("rtb_fused_mixed32_scheme", "k_fused_mixed32")}

    def by_index(plan, n_rays):
        """A plan's X, Y and flags at the rays' indices (its outputs are at
        the tracing slots)."""
        out = E.device_view(plan.rays()[1])
        order = plan.order(n_rays)
        if order is None:
            return out
        res = {}
        for k in ("X", "Y", "flag"):
            t = torch.empty_like(out[k])
            t[order] = out[k]
            res[k] = t
        return res

    def traced(st):
        # beams whose every ray is lost are reported (first one in stats), the
        # others traced: only a failure of the call itself stops the bench
        if st not in (ffi.OK, ffi.NO_INTERSECTIONS, ffi.NO_GOOD_RAYS):
            ffi.check(st, "rtb_plan_run")

    def timed_plan(plan, K, W):
        for _ in range(W):
            plan.run(C.c_void_p(stream.cuda_stream))
        traced(plan.result()[0])
        replicas.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            plan.run(C.c_void_p(stream.cuda_stream))
        e1.record(stream)
        torch.cuda.synchronize()
        ms = replicas.max_over_ranks(e0.elapsed_time(e1))
        st, stats = plan.result()
        traced(st)
        stats.rs = replicas.sum_over_ranks(stats.ray_surfaces)
        return ms / K, stats

    want = set(args.engines.split(","))
    head = None
    clocks = None
    plans = {}
    # the plain FP64 per-surface engine: one kernel per surface (rtb_trace_out)
    if "per_surface" in want:
        o = mk(ffi.ENGINE_PER_SURFACE, ffi.FP64)
        try:
            step(o)
            ms, stats = timed(o, max(2, args.steps // 4), 1)
            engines["per_surface"] = {"ms_per_step": ms, "value": stats.rs / (ms * 1e-3),
                                      "ray_surfaces_per_step": stats.ray_surfaces, "n_good": stats.n_good,
                                      "launch": "rtb_trace_out, 7 surface kernels + frame kernel"}
        except RuntimeError as e:
            engines["per_surface"] = {"error": str(e)}
    # the fused kernels: a plan each (rays generated in HBM once, one graph
    # launch per step, launch configuration from the autotuner), outputs
    # stored at the tracing slot (RTB_OUT_SLOT; rtb_plan_order maps them to
    # the rays)
    clocks_of = {}
    for name, prec in FUSED:
        if name not in want:
            continue
        try:
            torch.cuda.synchronize()
            t_create = time.perf_counter()
            plan = E.Plan(surf, beams, mk(ffi.ENGINE_FUSED, prec, out_order=ffi.OUT_SLOT))
            torch.cuda.synchronize()
            t_create = time.perf_counter() - t_create
            table = [] if args.no_autotune else plan.autotune(reps=2)
            block, rpt, _ = plan.config()
            if prec != ffi.FP64 or not (want & set(MIXED_ENGINES)):
                with Clocks(local) as ck:
                    ms, stats = timed_plan(plan, args.steps, args.warmup)
                clocks_of[name] = ck.summary()
            else:
                ms, stats = timed_plan(plan, max(2, args.steps // 4), 1)
            # the same plan storing at the rays' indices, and in index order:
            # what the slot-order stores and the coherent order gain
            variants = {}
            for key, ro, oo in (("index_outputs", ffi.ORDER_COHERENT, ffi.OUT_INDEX),
                                ("index_order", ffi.ORDER_INDEX, ffi.OUT_INDEX)):
                o_v = mk(ffi.ENGINE_FUSED, prec, out_order=oo)
                o_v.ray_order = ro
                p_v = E.Plan(surf, beams, o_v)
                ffi.check(p_v.set_config(block, rpt), "rtb_plan_set_config")
                ms_v, _ = timed_plan(p_v, max(2, args.steps // 4), 1)
                variants[key] = {"ms_per_step": ms_v, "value": stats.rs / (ms_v * 1e-3)}
                p_v.destroy()
        except RuntimeError as e:
            engines[name] = {"error": str(e)}
            continue
        plans[name] = plan
        cnt = plan.counts().sum(axis=0).astype(np.int64)  # per stage: rays lost there; last: rays at the end
        lost_before = np.concatenate([[0], np.cumsum(cnt[:-1])])
        reaching = [int(n - lost_before[3 * k]) for k in range(len(surf))]
        spec_on, spec_note = plan.specialized()
        kname, generic = KERNELS[prec]
        engines[name] = {"ms_per_step": ms, "value": stats.rs / (ms * 1e-3),
                         "kernel": (f"{kname} ({generic} compiled with NVRTC for the scheme when the plan is "
                                    "made: structure fixed, surface constants baked in)") if spec_on else generic,
                         "specialised": spec_on, "specialise_note": spec_note,
                         "ray_surfaces_per_step": stats.ray_surfaces, "n_good": stats.n_good,
                         "launch": f"rtb_plan_run (CUDA graph), block {block} x {rpt} rays/thread"
                                   + ("" if args.no_autotune else " (autotuned)"),
                         "ray_order": "coherent (beam, wavelength, Morton code of the entrance position), "
                                      "sorted once when the plan is made",
                         "outputs": "at the tracing slot (RTB_OUT_SLOT)",
                         "rays_reaching_surfaces": reaching,
                         "plan_create_s": t_create, **variants,
                         "autotune_ms": {f"{b}x{r}": round(t, 4) for b, r, t in table}}

    # accuracy of each mixed engine against the FP64 plan on the same rays
    # (the plans generate identical rays from the same beam table)
    accuracy = {}
    if "fused_fp64" in plans:
        from rt_b200 import metrics
        ref = by_index(plans["fused_fp64"], n)
        for name in MIXED_ENGINES:
            if name in plans:
                a = by_index(plans[name], n)
                accuracy[name] = metrics.ccd_error(a["X"], a["Y"], a["flag"], ref["X"], ref["Y"], ref["flag"],
                                                   ccd.xsize, ccd.ysize, ccd.xpix, ccd.ypix)
                engines[name]["accuracy_vs_fp64"] = accuracy[name]
    for p_ in plans.values():
        p_.destroy()
    plans.clear()
    # the headline: the faster mixed engine within 0.05 um at p99.9
    for name in MIXED_ENGINES:
        e = engines.get(name, {})
        ok = "value" in e and (name not in accuracy or accuracy[name].get("p99_9_um", 1e9) <= 0.05)
        if ok and (head is None or e["ms_per_step"] < engines[head]["ms_per_step"]):
            head = name
    if head is None and "value" in engines.get("fused_fp64", {}):
        head = "fused_fp64"
    clocks = clocks_of.get(head)
    if head is None and "value" in engines.get("per_surface", {}):
        head = "per_surface"
    if head is None:
        raise SystemExit("no engine ran")
    hv = engines[head]

    head_prec = PREC.get(head, ffi.FP64)
    # C3: 512 beams of uneven size, wavelength, field angle and order in one
    # graph launch of the headline kernel, launch configuration autotuned.
    # Most of C3's rays are lost early (random order x wavelength: 192 of the
    # 512 beams reach the CCD), so its ray-surfaces/s is not comparable with
    # C1's.
    c3 = None
    if not args.no_c3 and head in MIXED_ENGINES:
        b3 = S.c3_beams()
        plan = E.Plan(surf, b3, mk(ffi.ENGINE_FUSED, head_prec, out_order=ffi.OUT_SLOT))
        table = [] if args.no_autotune else plan.autotune(reps=3)
        block, rpt, n3 = plan.config()
        ms3, st3 = timed_plan(plan, args.steps, args.warmup)
        cnt = plan.counts()
        c3 = {"beams": len(b3), "n_rays": n3, "beams_with_good_rays": int((cnt[:, -1] > 0).sum()),
              "ray_surfaces_per_run": st3.ray_surfaces, "n_good": st3.n_good,
              "ms_per_run": ms3, "value": st3.rs / (ms3 * 1e-3), "unit": UNIT, "engine": head,
              "config": {"block_size": block, "rays_per_thread": rpt},
              "autotune_ms": {f"{b}x{r}": round(t, 4) for b, r, t in table},
              "note": "most rays are lost early (192 of 512 beams reach the CCD): not comparable with C1",
              "how": "rtb_plan_run: one CUDA graph (counter clear, fused kernel, counter copy) per run"}
        plan.destroy()

    # C4: the adjoint pair (gradient of the spot merit in 24 parameters)
    c4 = None
    if not args.no_c4:
        try:
            c4 = c4_adjoint(args.c4_rays_per_lambda)
        except RuntimeError as e:
            c4 = {"error": str(e)}

    # roofline of the headline kernel (HBM view): algorithmic bytes per launch
    # = its input rows (Row64: 57 B, Row32: 33 B per ray) + 18 B written per
    # ray (X, Y, flag, lost_stage at the tracing slot) + 4 B per ray counted
    # on the frame
    prof = KERNEL_PROFILE.get(head, {})
    in_bytes = ROW_BYTES_PER_RAY.get(head, 57 + 4)
    alg_bytes = n * (in_bytes + 18) + hv["n_good"] * 4
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = alg_bytes / (hv["ms_per_step"] * 1e-3) / 1e9
    tpr = prof.get("traffic_per_ray")
    traffic = tpr * n if tpr else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_per_ray_bytes": tpr, "alg_bytes": alg_bytes,
                "alg_bytes_per_ray": alg_bytes / n,
                "kernel": hv.get("kernel", "").split(" ")[0],
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this "
                                  "workload, per ray, times the rays of a step" if tpr else None,
                "note": "HBM view of a kernel bound by instruction issue (no FP64, FP32 or memory pipe "
                        "saturated): the compute roofline is roofline_fp64"}

    # compute roofline of the headline kernel.  Algorithmic flops: the
    # reference algorithm's operations per ray at each surface (the CPU
    # oracle on the counting scalar, oracle/count_flops.py ->
    # rt_b200/data/flops_c1.json) times the rays this step sent to that
    # surface; executed flops: ncu op counters of the kernel (KERNEL_PROFILE).
    # Peaks: cuBLAS DGEMM and SGEMM (TF32 off) measured in this run.
    fp64_peak, fp32_peak = dgemm_tflops(), sgemm_tflops()
    sec = hv["ms_per_step"] * 1e-3
    alg = None
    try:
        tab = json.load(open(os.path.join(ROOT, "rt_b200", "data", "flops_c1.json")))
        reach = hv.get("rays_reaching_surfaces")
        if reach and len(reach) == len(tab["surfaces"]) and not args.surfaces:
            alg = sum(r * row["ops_per_ray"] for r, row in zip(reach, tab["surfaces"]))
            alg += tab["lost_ray_renormalize_ops"] / tab["sample_rays"] * n
    except (OSError, KeyError, ValueError):
        alg = None
    f64pr, f32pr = prof.get("f64_flops_per_ray"), prof.get("f32_flops_per_ray")
    tf = lambda flops: flops / sec / 1e12 if flops else None  # noqa: E731
    frac = lambda a, p: (a / p) if (a and p) else None  # noqa: E731
    roofline_fp64 = {"bound": "fp64", "achieved": tf(alg), "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": frac(tf(alg), fp64_peak),
                     "alg_flops_per_ray": (alg / n) if alg else None,
                     "executed_flops_per_ray": f64pr,
                     "executed_achieved": tf(f64pr * n if f64pr else None),
                     "executed_frac": frac(tf(f64pr * n if f64pr else None), fp64_peak),
                     "f32_executed_flops_per_ray": f32pr,
                     "f32_executed_achieved": tf(f32pr * n if f32pr else None), "f32_peak": fp32_peak,
                     "f32_executed_frac": frac(tf(f32pr * n if f32pr else None), fp32_peak),
                     "peak_source": "cuBLAS DGEMM / SGEMM (TF32 off) 4096^3 measured in this run (best of 5)",
                     "note": "achieved = the reference algorithm's FP64 operations (oracle op count per "
                             "surface x rays reaching it) per second; executed = the kernel's own FP64 "
                             "operations (ncu, FMA = 2), Newton refinements of its reciprocals and square "
                             "roots included"}
    if "per_surface" in engines and "value" in engines["per_surface"]:
        ps = engines["per_surface"]
        gbs = ALG_BYTES_PER_RAY_SURFACE * ps["value"] / 1e9
        ps["hbm_roofline"] = {"achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak,
                              "bytes_per_ray_surface": ALG_BYTES_PER_RAY_SURFACE}

    e2e = None
    if not args.no_e2e:
        h = E.PinnedRays(n)
        src_cpu = {f: getattr(rays_in, f).cpu().numpy() for f in E.FIELDS}
        o = mk(ffi.ENGINE_FUSED, head_prec)
        # the kernel compiled for the scheme (cached from the plan above;
        # rtb_specialize is the call a user makes ahead of one-shot traces)
        st_s, note = E.specialize(surf, FIXES, o.precision)
        spec = KERNELS[head_prec][0] if st_s == ffi.OK else KERNELS[head_prec][1] + f" ({note})"
        times = []
        for it in range(2 + max(1, args.steps // 3)):
            for f in E.FIELDS:
                np.copyto(getattr(h, f), src_cpu[f])
            h.flag[:] = 1
            replicas.barrier()
            t0 = time.perf_counter()
            st, stats = E.trace_host(surf, beams, h, o)
            times.append(replicas.max_over_ranks(time.perf_counter() - t0))
            ffi.check(st, "rtb_trace_host")
        t = float(np.median(times[2:]))
        rs = replicas.sum_over_ranks(stats.ray_surfaces)
        n_all = replicas.sum_over_ranks(n)
        e2e = {"value": rs / t, "unit": UNIT, "h2d_bytes_per_step": int(n_all) * (7 * 8 + 1 + 1),
               "d2h_bytes_per_step": int(n_all) * (2 * 8 + 1 + 1), "seconds_per_step": t,
               "how": "rtb_trace_host on page-locked host arrays, wall clock (slowest rank), median of steps",
               "kernel": spec}
        h.free()

    cpu = None
    if not args.no_cpu and rank == 0:
        cpu = cpu_baseline(S.echelle, beams)

    if rank == 0:
        line = {"metric": METRIC, "value": hv["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": hv["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if head in MIXED_ENGINES else "f64",
                "data": "synthetic",
                "config": workload_config(n, len(beams)), "engine": head,
                "engines": engines,
                "speedup_vs_plain_fp64": (hv["value"] / engines["per_surface"]["value"])
                if "per_surface" in engines and "value" in engines["per_surface"] else None,
                "accuracy_vs_fp64": accuracy,
                "c3_batched": c3,
                "c4_adjoint": c4,
                "roofline": roofline, "roofline_fp64": roofline_fp64, "cpu_baseline": cpu, "e2e": e2e,
                "clocks": clocks,
                "gpu_launches": args.steps * 1}
        print(json.dumps(line), flush=True)
    replicas.finish()


if __name__ == "__main__":
    main()
