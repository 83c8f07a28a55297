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
