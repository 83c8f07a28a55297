"""rtb_trace_out_noalloc: the fused trace for callers that cannot allocate.

Some callers cannot let a library allocate device memory: their own
allocator has reserved the device memory up front, or they run under a fixed
memory budget where no allocator may be called.  rtb_trace_out_noalloc keeps
the fused kernel's scratch in a fixed 1 MiB device array instead.  These GPU
tests call it through the C ABI and check that two calls in a row give what
rtb_trace_out gives on the same inputs (bit for bit: the same generic kernel
runs on the same rays, with the scheme prepared by the same code), and that
requests beyond its limits are refused.  The file
is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu


def _bind():
    L = E.lib()
    for name in ("rtb_trace_out", "rtb_trace_out_noalloc"):
        fn = getattr(L, name)
        fn.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                       C.POINTER(ffi.TraceOpts), C.POINTER(ffi.Rays), C.POINTER(ffi.Rays),
                       C.POINTER(ffi.TraceStats), C.c_void_p]
    return L


def _call(fn, surfaces, beams, o, rin, rout):
    s_arr = (ffi.Surface * len(surfaces))(*surfaces)
    b_arr = (ffi.Beam * len(beams))(*beams)
    stats = ffi.TraceStats()
    st = fn(s_arr, len(surfaces), b_arr, len(beams), C.byref(o), C.byref(rin.struct()), C.byref(rout.struct()),
            C.byref(stats), None)
    torch.cuda.synchronize()
    return st, stats


def _same(a, b):
    for f in E.FIELDS[:6] + ("flag", "lost_stage"):
        x, y = getattr(a, f), getattr(b, f)
        if x.dtype == torch.float64:
            eq = (x.view(torch.int64) == y.view(torch.int64)) | (torch.isnan(x) & torch.isnan(y))
        else:
            eq = x == y
        assert bool(eq.all()), f


@pytest.mark.parametrize("precision", [ffi.FP64, ffi.MIXED])
def test_noalloc_matches_trace_out_on_two_calls(precision, monkeypatch):
    # rtb_trace_out_noalloc runs the generic fused kernels; rtb_trace_out
    # would launch a kernel compiled for the scheme if an earlier test had
    # compiled one, and the mixed one folds the scheme's constants into its
    # arithmetic (a few ulps apart): compare with the generic kernels
    monkeypatch.setenv("RTB_SPECIALIZE", "0")
    L = _bind()
    cases = [
        (S.echelle(), S.c1_beams(n_per_lambda=120)[:6], 3),      # several beams with per-beam orders
        (S.littrow_free(), S.c0_beams(n_per_lambda=3000), 0),    # smaller scheme: leftovers must not leak
        # wavelengths on the knots of the lens glass's uniform grid (0.35 + 0.01 i):
        # the table lookups of both entry points must pick the same intervals
        (S.echelle(), [S.make_beam(0, 200, 51, S.C1_RADIUS, (0.40, 0.90), 7, orders=(40, 1))], 3),
    ]
    for specs, beams, fixes in cases:
        cs = S.to_c(specs, E.spline_init)
        n = S.total_rays(beams)
        rin = E.generate(beams, n)
        out_ref, out_na = E.DeviceRays(n), E.DeviceRays(n)
        o = E.opts(engine=ffi.ENGINE_FUSED, precision=precision, fixes=fixes)
        st_r, stats_r = _call(L.rtb_trace_out, cs.surfaces, beams, o, rin, out_ref)
        for _ in range(2):  # the second call must not see the first one's scratch
            st_n, stats_n = _call(L.rtb_trace_out_noalloc, cs.surfaces, beams, o, rin, out_na)
            assert st_r == st_n == ffi.OK
            assert (stats_n.ray_surfaces, stats_n.n_good, stats_n.failed_beam, stats_n.failed_stage) == \
                (stats_r.ray_surfaces, stats_r.n_good, stats_r.failed_beam, stats_r.failed_stage)
            _same(out_na, out_ref)


def test_noalloc_rejects_requests_beyond_its_limit():
    L = _bind()
    specs = S.echelle()
    cs = S.to_c(specs, E.spline_init)
    too_many = 1_000_000 // (8 * (3 * len(specs) + 1)) + 10   # loss counters alone exceed the array
    beams = [S.make_beam(i, 1, 1, 1.0, (0.5, 0.5), i) for i in range(too_many)]
    rin = E.DeviceRays(too_many)
    out = E.DeviceRays(too_many)
    st, _ = _call(L.rtb_trace_out_noalloc, cs.surfaces, beams, E.opts(), rin, out)
    assert st == ffi.BAD_VALUE
    o = E.opts(engine=ffi.ENGINE_PER_SURFACE)
    st, _ = _call(L.rtb_trace_out_noalloc, cs.surfaces, beams[:1], o, rin, out)
    assert st == ffi.BAD_VALUE
    # launch configurations rtb_trace_out refuses are refused here too
    for block, rpt in ((96, 2), (512, 2), (256, 65)):
        o = E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64)
        o.block_size, o.rays_per_thread = block, rpt
        st, _ = _call(L.rtb_trace_out_noalloc, cs.surfaces, beams[:1], o, rin, out)
        assert st == ffi.BAD_VALUE, (block, rpt)
