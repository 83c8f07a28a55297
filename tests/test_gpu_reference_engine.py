"""The reference's own CUDA engine on the same B200, timed beside this one
(GPU test; skipped when oracle/_ref/harness_refgpu is not built).

oracle/_ref/harness_refgpu is the reference's Beam/Surface/TabulatedFunction
host classes over its cuda_engine compiled for sm_100a (oracle/Makefile),
driving Scheme::run's surface loop (scheme.cpp:983-1055) with its host
copies per engine call.  One C1 order range (order 45, 64 wavelengths x
50404 rays = 3.2e6 rays, the reference's quirks as they are: fixes 0) goes
through it (an eighth of the range with the toric fold unless RTB_REF_FULL=1)
and through this library: the per-surface FP64 engine on rays in
HBM, the same engine on host arrays (rtb_trace_host, copies included) and the
fused mixed kernel.  The test prints the times; it checks that this engine's
FP64 result has the reference's number of good rays to within the rays the
toric 0/0 and FMA contraction decide differently, and that it is faster.
"""
import ctypes as C
import json
import os
import re
import subprocess
import tempfile
import time

import numpy as np
import pytest
import torch

import pyoracle as O
import refharness as H
from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu


def sphere_fold(specs):
    """C1 with the toric fold replaced by a sphere of the mean radius: the
    reference's iter_toric prints from the device for every ray
    (rt_cuda_engine_surface.cu:359-410), which dominates its time."""
    out = []
    for s in specs:
        s = S.SurfaceSpec(**s.__dict__)
        if s.cls == ffi.TORIC:
            s.cls, s.params = ffi.CONIC, (-1 / 2050.0, 0.0, 0)
        out.append(s)
    return out


@pytest.mark.skipif(H.harness("refgpu") is None, reason="reference cuda_engine harness not built")
@pytest.mark.parametrize("variant", ["c1", "c1_sphere_fold"])
def test_reference_cuda_engine_speed(variant):
    specs = S.echelle() if variant == "c1" else sphere_fold(S.echelle())
    # the reference needs ~140 s for the full range with the toric: an eighth
    # of it by default, the full range with RTB_REF_FULL=1
    n_per = S.c1_rays_per_lambda()
    if variant == "c1" and os.environ.get("RTB_REF_FULL") != "1":
        n_per //= 8
    beam = S.make_beam(0, n_per, S.C1_NLAMBDA, S.C1_RADIUS, S.C1_LAMBDA, S.SEED + 45, orders=(45, 1))
    n = beam.n_rays
    rays = O.generate([beam], n)
    with tempfile.TemporaryDirectory() as d:
        spec = H.write_spec(specs, [45, 1], d)
        bin_path = H.write_beam(rays, d)
        out = subprocess.run([H.harness("refgpu"), "trace", spec, bin_path, d + "/out.dat"], capture_output=True,
                             text=True, timeout=1200)
    m = re.search(r"trace_seconds=([0-9.]+) good=(\d+)", out.stderr)
    assert out.returncode in (0, 5, 6) and m, out.stderr[-2000:]
    ref_s, ref_good = float(m.group(1)), int(m.group(2))

    cs = S.to_c(specs, E.spline_init)
    dev = E.DeviceRays.from_host(rays)
    torch.cuda.synchronize()
    res = {}
    for name, o in (("per_surface_fp64", E.opts(engine=ffi.ENGINE_PER_SURFACE, precision=ffi.FP64, state_out=0)),
                    ("fused_mixed", E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, state_out=0))):
        best = 1e9
        for _ in range(3):
            r = dev.copy()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st, stats = E.trace(cs.surfaces, [beam], r, o)
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        res[name] = (best, stats.n_good, stats.ray_surfaces)
    h = E.PinnedRays(n)
    for f in E.FIELDS:
        getattr(h, f)[:] = getattr(rays, f)
    t0 = time.perf_counter()
    st, stats = E.trace_host(cs.surfaces, [beam], h, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, state_out=0))
    res["host_arrays_fused_fp64"] = (time.perf_counter() - t0, stats.n_good, stats.ray_surfaces)
    h.free()
    rs = res["per_surface_fp64"][2]
    line = {"variant": variant, "rays": n, "ray_surfaces": rs, "reference_cuda_engine_s": ref_s, "reference_good": ref_good,
            "reference_rate": rs / ref_s}
    for k, (t, g, r_s) in res.items():
        line[k + "_s"] = t
        line[k + "_rate"] = r_s / t
        line[k + "_good"] = g
    print(json.dumps(line))
    if variant == "c1_sphere_fold":  # no toric 0/0: the same rays survive, FMA contraction aside
        assert abs(res["per_surface_fp64"][1] - ref_good) <= 1e-4 * n
    else:
        assert abs(res["per_surface_fp64"][1] - ref_good) <= 0.3 * n
    assert res["per_surface_fp64"][0] < ref_s


@pytest.mark.skipif(os.environ.get("RTB_REF_C1") != "1", reason="minutes of GPU time: set RTB_REF_C1=1")
@pytest.mark.skipif(H.harness("refgpu") is None or H.harness("refgpu_ptx") is None,
                    reason="reference cuda_engine harnesses not built")
def test_reference_cuda_engine_whole_c1(tmp_path):
    """The reference's cuda_engine over the whole C1 workload -- all 31 echelle
    order ranges, 1.0e8 rays, the fold as a sphere (with the toric, its
    per-ray device printf and cycling rays take ~140 s per range) -- built as
    the reference ships it (compute_50 PTX, compiled by the driver at load,
    CMakeLists.txt:115) and for sm_100a, each range through Scheme::run's
    loop in its own process as the reference runs ranges; this engine's
    per-surface FP64, fused FP64 and fused mixed paths on the same rays, with
    the SM clocks sampled meanwhile.  Prints one JSON line and writes it to
    $RTB_REF_C1_OUT when set."""
    from rt_b200.clocks import Clocks
    specs = sphere_fold(S.echelle())
    beams = S.c1_beams()
    n = S.total_rays(beams)
    line = {"workload": "C1, fold as a sphere: 31 ranges (orders 30..60) x 64 wavelengths x 50404 rays",
            "rays": n, "builds": {}}
    spec_dir = str(tmp_path)
    for kind, label in (("refgpu_ptx", "compute_50 PTX as shipped, JIT"), ("refgpu", "sm_100a")):
        total_s, good, per_range = 0.0, 0, []
        with Clocks(0) as ck:
            for b in beams:
                m = int(b.orders[0])
                one = S.make_beam(0, int(b.disk[0]), S.C1_NLAMBDA, S.C1_RADIUS, S.C1_LAMBDA, int(b.seed),
                                  orders=(m, 1))
                rays = O.generate([one], one.n_rays)
                spec = H.write_spec(specs, [m, 1], spec_dir)
                bin_path = H.write_beam(rays, spec_dir)
                out = subprocess.run([H.harness(kind), "trace", spec, bin_path, spec_dir + "/out.dat"],
                                     capture_output=True, text=True, timeout=600)
                mm = re.search(r"trace_seconds=([0-9.]+) good=(\d+)", out.stderr)
                assert out.returncode in (0, 5, 6) and mm, out.stderr[-2000:]
                total_s += float(mm.group(1))
                good += int(mm.group(2))
                per_range.append(round(float(mm.group(1)), 4))
        line["builds"][label] = {"trace_seconds": total_s, "good": good, "per_range_s": per_range,
                                 "clocks": ck.summary()}
    # this engine on the same rays (one call or one plan run for all ranges)
    cs = S.to_c(specs, E.spline_init)
    rays = E.generate(beams, n)
    ours = {}
    o_ps = E.opts(engine=ffi.ENGINE_PER_SURFACE, precision=ffi.FP64, state_out=0)
    best = 1e9
    for _ in range(3):
        r = rays.copy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, stats = E.trace(cs.surfaces, beams, r, o_ps)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
        del r
    rs, ours["per_surface_fp64"] = stats.ray_surfaces, {"seconds": best, "good": stats.n_good}
    for name, prec in (("fused_fp64", ffi.FP64), ("fused_mixed", ffi.MIXED), ("fused_mixed32", ffi.MIXED32)):
        plan = E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=prec, state_out=0,
                                                  out_order=ffi.OUT_SLOT))
        plan.run()
        plan.result()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(5):
            plan.run()
        st, stats = plan.result()
        ours[name] = {"seconds": (time.perf_counter() - t0) / 5, "good": stats.n_good}
        plan.destroy()
    line["ray_surfaces"] = rs
    for k, v in line["builds"].items():
        v["rate"] = rs / v["trace_seconds"]
    for k, v in ours.items():
        v["rate"] = rs / v["seconds"]
    line["this_engine"] = ours
    print(json.dumps(line))
    if os.environ.get("RTB_REF_C1_OUT"):
        with open(os.environ["RTB_REF_C1_OUT"], "w") as f:
            f.write(json.dumps(line) + "\n")
    sm = line["builds"]["sm_100a"]
    assert abs(ours["per_surface_fp64"]["good"] - sm["good"]) <= 1e-4 * n
    assert ours["per_surface_fp64"]["seconds"] < sm["trace_seconds"]
