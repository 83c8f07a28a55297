"""Failures made on the host, and the status codes they come back as.

Nothing here faults a GPU.  The failures are made on the host: result files
cut short or missing (the reference's load_beam_data returns its read errors,
beam.cpp:829-1036), schemes with NaN or infinite numbers, and device
allocations made to fail by the library's fault hook
(rtb_fail_allocations), which the calls must report as RTB_BAD_ALLOC
(the reference's ENGINE_ERROR_BAD_ALLOC, rt_engine_errors.h:4) without
leaking what they had allocated before the failure.
"""
import ctypes as C
import math
import os
import struct

import numpy as np
import pytest

import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S


def _write_dat(path, n, n_good, n_lambda, arrays):
    """A result file in the reference's layout (beam.cpp:636-715): n, n_good,
    n_lambda as size_t, then X..lambda of the good rays, then of the rest."""
    with open(path, "wb") as f:
        f.write(struct.pack("<3Q", n, n_good, n_lambda))
        for part in (slice(0, n_good), slice(n_good, n)):
            for a in arrays:
                f.write(np.ascontiguousarray(a[part], dtype=np.float64).tobytes())


def _bind():
    L = ffi.load()
    L.rtb_read_dat_header.argtypes = [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_uint64)]
    L.rtb_read_dat.argtypes = [C.c_char_p, C.POINTER(ffi.Rays)]
    L.rtb_fail_allocations.argtypes = [C.c_uint32, C.c_uint32]
    return L


def _host_rays(n):
    arrs = {f: np.zeros(n) for f in ("X", "Y", "Z", "cX", "cY", "cZ", "lambda_")}
    flag = np.zeros(n, dtype=np.int8)
    r = ffi.Rays()
    for f, a in arrs.items():
        setattr(r, f, a.ctypes.data)
    r.flag = flag.ctypes.data
    r.lost_stage = None
    r.n = n
    return r, arrs, flag


def test_truncated_and_missing_result_files(tmp_path):
    L = _bind()
    n, ng = 100, 60
    rng = np.random.default_rng(3)
    arrays = [rng.normal(size=n) for _ in range(7)]
    path = str(tmp_path / "full.dat")
    _write_dat(path, n, ng, 5, arrays)
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    assert L.rtb_read_dat_header(path.encode(), C.byref(a), C.byref(b), C.byref(c)) == ffi.OK
    assert (a.value, b.value, c.value) == (n, ng, 5)
    r, arrs, flag = _host_rays(n)
    assert L.rtb_read_dat(path.encode(), C.byref(r)) == ffi.OK
    assert np.array_equal(arrs["X"][:ng], arrays[0][:ng]) and np.array_equal(arrs["lambda_"][ng:], arrays[6][ng:])
    assert flag.tolist() == [1] * ng + [0] * (n - ng)
    full = open(path, "rb").read()
    # cut inside the header, inside the good rays, inside the lost rays, one byte short
    for cut in (5, 24 + 8 * ng * 3 + 4, 24 + 8 * (7 * ng + 10), len(full) - 1):
        short = str(tmp_path / f"cut{cut}.dat")
        with open(short, "wb") as f:
            f.write(full[:cut])
        r, _, _ = _host_rays(n)
        assert L.rtb_read_dat(short.encode(), C.byref(r)) == ffi.BAD_VALUE, cut
        if cut < 24:
            assert L.rtb_read_dat_header(short.encode(), C.byref(a), C.byref(b), C.byref(c)) == ffi.BAD_VALUE
    # a header whose good count exceeds its ray count, a ray count other than the arrays'
    bad = str(tmp_path / "bad.dat")
    with open(bad, "wb") as f:
        f.write(struct.pack("<3Q", 10, 11, 1))
    assert L.rtb_read_dat_header(bad.encode(), C.byref(a), C.byref(b), C.byref(c)) == ffi.BAD_VALUE
    r, _, _ = _host_rays(n - 1)
    assert L.rtb_read_dat(path.encode(), C.byref(r)) == ffi.BAD_VALUE
    # no file
    missing = str(tmp_path / "none.dat").encode()
    assert L.rtb_read_dat_header(missing, C.byref(a), C.byref(b), C.byref(c)) == ffi.FAILED
    r, _, _ = _host_rays(n)
    assert L.rtb_read_dat(missing, C.byref(r)) == ffi.FAILED


def _nonfinite_schemes():
    """C1 with one number of one surface made NaN or infinite, each way."""
    out = []
    for k, field, idx in ((0, "params", 0), (4, "params", 5), (3, "params", 3), (1, "distance", 2),
                          (2, "angles", 1), (5, "size", 0), (1, "gr_const", None)):
        for bad in (math.nan, math.inf, -math.inf):
            specs = S.echelle()
            s = specs[k]
            if idx is None:
                setattr(s, field, bad)
            else:
                v = list(getattr(s, field))
                v[idx] = bad
                setattr(s, field, tuple(v))
            out.append((f"{field}[{idx}] of surface {k} = {bad}", specs))
    return out


def test_nonfinite_scheme_numbers_are_refused_before_any_launch():
    """rtb_specialize prepares the scheme exactly as a trace does, without a
    device: a NaN or infinity in any number a trace uses is RTB_BAD_VALUE."""
    for what, specs in _nonfinite_schemes():
        cs = S.to_c(specs, O.spline_init)
        st, _ = E.specialize(list(cs.surfaces), 3, ffi.MIXED)
        assert st == ffi.BAD_VALUE, what
    st, note = E.specialize(list(S.to_c(S.echelle(), O.spline_init).surfaces), 3, ffi.MIXED)
    assert st == ffi.OK, note


@pytest.mark.gpu
def test_nonfinite_scheme_numbers_refused_by_traces_and_plans():
    import torch
    beams = S.c1_beams(n_per_lambda=10)[:2]
    n = S.total_rays(beams)
    rays = E.generate(beams, n)
    for what, specs in _nonfinite_schemes()[::3]:
        cs = S.to_c(specs, E.spline_init)
        st, _ = E.trace(cs.surfaces, beams, rays.copy(), E.opts(precision=ffi.MIXED, fixes=3))
        assert st == ffi.BAD_VALUE, what
        with pytest.raises(RuntimeError, match="BAD_VALUE"):
            E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED32, fixes=3))
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_allocation_failures_are_reported_and_leak_nothing():
    """Each device allocation of a trace and of a plan, failing in turn: the
    call returns RTB_BAD_ALLOC, the next call succeeds, and the device memory
    in use is what it was before."""
    import torch
    L = _bind()
    L.rtb_trace_out.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                                C.POINTER(ffi.TraceOpts), C.POINTER(ffi.Rays), C.POINTER(ffi.Rays),
                                C.POINTER(ffi.TraceStats), C.c_void_p]
    beams = S.c1_beams(n_per_lambda=50)[:4]
    n = S.total_rays(beams)
    cs = S.to_c(S.echelle(), E.spline_init)
    surf = (ffi.Surface * len(cs.surfaces))(*cs.surfaces)
    rin, rout = E.generate(beams, n), E.DeviceRays(n)
    o = E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=3)

    def trace():
        stats = ffi.TraceStats()
        st = L.rtb_trace_out(surf, len(surf), E._beams(beams), len(beams), C.byref(o), C.byref(rin.struct()),
                             C.byref(rout.struct()), C.byref(stats), None)
        torch.cuda.synchronize()
        return st

    def plan():
        p = C.c_void_p()
        po = E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED32, fixes=3)
        st = L.rtb_plan_create(surf, len(surf), E._beams(beams), len(beams), C.byref(po), C.byref(p))
        if st == ffi.OK:
            L.rtb_plan_run(p, None)
            st2 = L.rtb_plan_result(p, C.byref(ffi.TraceStats()))
            L.rtb_plan_destroy(p)
            assert st2 == ffi.OK
        return st

    for call in (trace, plan):
        L.rtb_fail_allocations(0, 0)
        assert call() == ffi.OK  # warm: pools, compiled kernels
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        failed = 0
        for after in range(8):  # the first, second, ... allocation of the call fails
            L.rtb_fail_allocations(after, 1)
            st = call()
            L.rtb_fail_allocations(0, 0)
            assert st in (ffi.BAD_ALLOC, ffi.OK), (call.__name__, after, st)
            failed += st == ffi.BAD_ALLOC
            assert call() == ffi.OK, (call.__name__, after)
        assert failed >= (1 if call is trace else 4), (call.__name__, failed)
        torch.cuda.synchronize()
        assert abs(torch.cuda.mem_get_info()[0] - free0) < (64 << 20), call.__name__
