"""Python driver of librtb200.so: device-resident rays and the trace calls.

Device memory comes from torch (allocation and streams only); every
computation is a call into the CUDA library through include/rtb.h.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ffi

FIELDS = ("X", "Y", "Z", "cX", "cY", "cZ", "lambda_")

_bound = False


def lib() -> C.CDLL:
    global _bound
    L = ffi.load()
    if not _bound:
        P = C.POINTER
        vp = C.c_void_p
        L.rtb_trace.argtypes = [P(ffi.Surface), C.c_size_t, P(ffi.Beam), C.c_size_t, P(ffi.TraceOpts), P(ffi.Rays),
                                P(ffi.TraceStats), vp]
        L.rtb_trace_host.argtypes = [P(ffi.Surface), C.c_size_t, P(ffi.Beam), C.c_size_t, P(ffi.TraceOpts),
                                     P(ffi.Rays), P(ffi.TraceStats)]
        L.rtb_generate_beams.argtypes = [P(ffi.Beam), C.c_size_t, P(ffi.Rays), vp]
        L.rtb_ccd_frame.argtypes = [P(ffi.Rays), P(ffi.CCD), vp, vp, vp]
        L.rtb_reference_order.argtypes = [P(ffi.Beam), C.c_size_t, C.c_size_t, P(ffi.Rays), vp, vp]
        L.rtb_spline_init.argtypes = [C.c_size_t, vp, vp, vp]
        L.rtb_info.argtypes = [C.c_char_p, C.c_size_t]
        L.rtb_alocate_vector.restype = P(C.c_double)
        L.rtb_alocate_vector.argtypes = [C.c_size_t]
        L.rtb_free_vector.argtypes = [P(C.c_double)]
        _bound = True
    return L


def spline_init(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Natural-spline second derivatives (rtb_spline_init, host code)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    y2 = np.zeros_like(x)
    ffi.check(lib().rtb_spline_init(len(x), ffi.vptr(x), ffi.vptr(y), ffi.vptr(y2)), "rtb_spline_init")
    return y2


def info() -> str:
    buf = C.create_string_buffer(1024)
    ffi.check(lib().rtb_info(buf, 1024), "rtb_info")
    return buf.value.decode()


class DeviceRays:
    """SoA ray arrays on the current CUDA device (torch tensors)."""

    def __init__(self, n: int, device="cuda"):
        import torch
        self.n = n
        for f in FIELDS:
            setattr(self, f, torch.empty(n, dtype=torch.float64, device=device))
        self.flag = torch.ones(n, dtype=torch.int8, device=device)
        self.lost_stage = torch.full((n,), ffi.NOT_LOST, dtype=torch.uint8, device=device)

    def struct(self) -> ffi.Rays:
        return ffi.Rays(*(ffi.vptr(getattr(self, f)) for f in FIELDS), ffi.vptr(self.flag),
                        ffi.vptr(self.lost_stage), self.n)

    @classmethod
    def from_host(cls, h) -> "DeviceRays":
        import torch
        d = cls(h.n)
        for f in FIELDS + ("flag", "lost_stage"):
            getattr(d, f).copy_(torch.from_numpy(np.ascontiguousarray(getattr(h, f))))
        return d

    def to_host(self, cls):
        h = cls(self.n)
        for f in FIELDS + ("flag", "lost_stage"):
            getattr(h, f)[:] = getattr(self, f).cpu().numpy()
        return h

    def copy(self) -> "DeviceRays":
        d = DeviceRays.__new__(DeviceRays)
        d.n = self.n
        for f in FIELDS + ("flag", "lost_stage"):
            setattr(d, f, getattr(self, f).clone())
        return d


def _beams(beams):
    return (ffi.Beam * len(beams))(*beams)


def generate(beams, n: int, stream=None) -> DeviceRays:
    rays = DeviceRays(n)
    st = lib().rtb_generate_beams(_beams(beams), len(beams), C.byref(rays.struct()), stream)
    ffi.check(st, "rtb_generate_beams")
    return rays


def opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, fixes=0, renorm_lost=1, state_out=1, block=0, rpt=0,
         ccd=None, counts=None, n_outside=None) -> ffi.TraceOpts:
    o = ffi.TraceOpts()
    o.engine, o.precision, o.fixes, o.renormalize_lost = engine, precision, fixes, renorm_lost
    o.block_size, o.rays_per_thread, o.state_out = block, rpt, state_out
    if ccd is not None:
        o._ccd = ccd  # keep alive
        o.ccd = C.pointer(ccd)
        o.counts = ffi.vptr(counts)
        o.n_outside = ffi.vptr(n_outside)
    return o


def trace(surfaces, beams, rays: DeviceRays, o: ffi.TraceOpts | None = None, stream=None):
    """In-place trace; returns (status, TraceStats)."""
    o = o or opts()
    surf = (ffi.Surface * len(surfaces))(*surfaces)
    stats = ffi.TraceStats()
    st = lib().rtb_trace(surf, len(surfaces), _beams(beams), len(beams), C.byref(o), C.byref(rays.struct()),
                         C.byref(stats), stream)
    return st, stats


def trace_host(surfaces, beams, host_rays, o: ffi.TraceOpts | None = None):
    o = o or opts()
    surf = (ffi.Surface * len(surfaces))(*surfaces)
    stats = ffi.TraceStats()
    st = lib().rtb_trace_host(surf, len(surfaces), _beams(beams), len(beams), C.byref(o),
                              C.byref(host_rays.struct()), C.byref(stats))
    return st, stats


def ccd_frame(rays: DeviceRays, ccd: ffi.CCD, counts=None, n_outside=None):
    import torch
    if counts is None:
        counts = torch.zeros(int(ccd.xdim) * int(ccd.ydim), dtype=torch.int32, device="cuda")
    if n_outside is None:
        n_outside = torch.zeros(1, dtype=torch.int64, device="cuda")
    st = lib().rtb_ccd_frame(C.byref(rays.struct()), C.byref(ccd), ffi.vptr(counts), ffi.vptr(n_outside), None)
    ffi.check(st, "rtb_ccd_frame")
    return counts, n_outside


def reference_order(beams, n_stages: int, rays: DeviceRays):
    import torch
    order = torch.empty(rays.n, dtype=torch.int32, device="cuda")
    st = lib().rtb_reference_order(_beams(beams), len(beams), n_stages, C.byref(rays.struct()), ffi.vptr(order), None)
    ffi.check(st, "rtb_reference_order")
    return order


class PinnedRays:
    """Host ray arrays in page-locked memory (rtb_alocate_vector)."""

    def __init__(self, n: int):
        self.n = n
        self._ptrs = []
        for f in FIELDS:
            p = lib().rtb_alocate_vector(n)
            if not p:
                raise MemoryError("rtb_alocate_vector failed")
            self._ptrs.append(p)
            setattr(self, f, np.ctypeslib.as_array(p, shape=(n,)))
        self.flag = np.ones(n, dtype=np.int8)
        self.lost_stage = np.full(n, ffi.NOT_LOST, dtype=np.uint8)

    def struct(self) -> ffi.Rays:
        return ffi.Rays(*(ffi.vptr(getattr(self, f)) for f in FIELDS), ffi.vptr(self.flag),
                        ffi.vptr(self.lost_stage), self.n)

    def free(self):
        for p in self._ptrs:
            lib().rtb_free_vector(p)
        self._ptrs = []
        for f in FIELDS:
            setattr(self, f, None)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
