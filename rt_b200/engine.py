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
        L.rtb_plan_create.argtypes = [P(ffi.Surface), C.c_size_t, P(ffi.Beam), C.c_size_t, P(ffi.TraceOpts),
                                      P(vp)]
        L.rtb_plan_run.argtypes = [vp, vp]
        L.rtb_plan_result.argtypes = [vp, P(ffi.TraceStats)]
        L.rtb_plan_rays.argtypes = [vp, P(ffi.Rays), P(ffi.Rays)]
        L.rtb_plan_order.argtypes = [vp, P(vp)]
        L.rtb_plan_counts.argtypes = [vp, vp, C.c_size_t, P(C.c_size_t)]
        L.rtb_plan_autotune.argtypes = [vp, C.c_int, P(ffi.TuneEntry), C.c_size_t, P(C.c_size_t)]
        L.rtb_plan_set_config.argtypes = [vp, C.c_int32, C.c_int32]
        L.rtb_plan_config.argtypes = [vp, P(C.c_int32), P(C.c_int32), P(C.c_uint64)]
        L.rtb_plan_destroy.argtypes = [vp]
        L.rtb_plan_specialized.argtypes = [vp, P(C.c_int32), C.c_char_p, C.c_size_t]
        L.rtb_specialize.argtypes = [P(ffi.Surface), C.c_size_t, C.c_uint32, C.c_int32, C.c_char_p, C.c_size_t]
        L.rtb_adjoint_specialize.argtypes = [P(ffi.Surface), C.c_size_t, C.c_uint32, C.c_char_p, C.c_size_t]
        L.rtb_adjoint_create.argtypes = [P(ffi.Surface), C.c_size_t, P(ffi.Param), C.c_size_t, P(ffi.Beam),
                                         C.c_size_t, C.c_uint64, C.c_uint32, P(vp)]
        L.rtb_adjoint_theta.argtypes = [vp, vp]
        L.rtb_adjoint_forward.argtypes = [vp, vp, P(ffi.Rays), vp, vp, vp, P(ffi.TraceStats), vp]
        L.rtb_adjoint_backward.argtypes = [vp, vp, vp, vp, vp]
        L.rtb_adjoint_jvp.argtypes = [vp, vp, vp, vp, vp]
        L.rtb_adjoint_spot_merit.argtypes = [vp, vp, C.c_double, P(C.c_double), vp, vp, vp]
        L.rtb_adjoint_resolution_merit.argtypes = [vp, vp, C.c_double, C.c_double, P(C.c_double), vp, vp, vp]
        L.rtb_adjoint_destroy.argtypes = [vp]
        L.rtb_qe_curves.argtypes = [P(ffi.QeSurface), C.c_size_t, vp, C.c_size_t, C.c_size_t, C.c_size_t, vp, vp]
        L.rtb_grating_energy_distr.argtypes = [C.c_size_t, vp, C.c_long] + [C.c_double] * 6 + [vp]
        L.rtb_surface_QE.argtypes = [C.c_size_t, vp, vp, P(ffi.Table)]
        L.rtb_loss_ratios.argtypes = [vp, C.c_uint64, C.c_uint64, C.c_uint64, vp, vp, vp]
        L.rtb_unique_lambdas.argtypes = [vp, C.c_uint64, C.c_uint64, vp, P(C.c_uint64), vp]
        _bound = True
    return L


def spline_init(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Natural-spline second derivatives (rtb_spline_init, host code)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    y2 = np.zeros_like(x)
    ffi.check(lib().rtb_spline_init(len(x), ffi.vptr(x), ffi.vptr(y), ffi.vptr(y2)), "rtb_spline_init")
    return y2


def qe_curves(cqe, rows, n_lambda: int) -> tuple[np.ndarray, np.ndarray]:
    """Scheme::ComputeQE's curves on the GPU (rtb_qe_curves, one launch) for
    the QE surfaces of `cqe` (schemes.CQe) over the wavelength-range rows:
    (lambda, qe), each n_rows x n_lambda."""
    rows = np.ascontiguousarray(np.atleast_2d(rows), dtype=np.float64)
    lam = np.zeros((rows.shape[0], n_lambda))
    qe = np.zeros_like(lam)
    ffi.check(lib().rtb_qe_curves(cqe.array, len(cqe), ffi.vptr(rows), rows.shape[0], rows.shape[1], n_lambda,
                                  ffi.vptr(lam), ffi.vptr(qe)), "rtb_qe_curves")
    return lam, qe


def loss_ratios(lam, n_good: int, n_lambda: int):
    """losses_comp's (ll, ratio) from a device tensor of wavelengths (good
    rays first), on the GPU (rtb_loss_ratios)."""
    ll, ratio = np.zeros(n_lambda), np.zeros(n_lambda)
    ffi.check(lib().rtb_loss_ratios(ffi.vptr(lam), lam.numel(), n_good, n_lambda, ffi.vptr(ll), ffi.vptr(ratio),
                                    None), "rtb_loss_ratios")
    return ll, ratio


def unique_lambdas(lam, n_good: int, max_out: int):
    """print_lambda's distinct wavelengths of lam[:n_good] (device tensor) in
    order of first occurrence, at most max_out (rtb_unique_lambdas)."""
    out = np.zeros(max(1, max_out))
    n = C.c_uint64(0)
    ffi.check(lib().rtb_unique_lambdas(ffi.vptr(lam), n_good, max_out, ffi.vptr(out), C.byref(n), None),
              "rtb_unique_lambdas")
    return out[:n.value].copy()


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
    """Seeded rays of `beams` on the device.  Without a stream the generator
    runs on the library's own stream, which is not ordered with torch's, so
    the call waits for it: the rays are complete when it returns."""
    rays = DeviceRays(n)
    st = lib().rtb_generate_beams(_beams(beams), len(beams), C.byref(rays.struct()), stream)
    ffi.check(st, "rtb_generate_beams")
    if stream is None:
        import torch
        torch.cuda.synchronize()
    return rays


def opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, fixes=0, renorm_lost=1, state_out=1, block=0, rpt=0,
         ccd=None, counts=None, n_outside=None, out_order=ffi.OUT_INDEX) -> ffi.TraceOpts:
    o = ffi.TraceOpts()
    o.engine, o.precision, o.fixes, o.renormalize_lost = engine, precision, fixes, renorm_lost
    o.block_size, o.rays_per_thread, o.state_out = block, rpt, state_out
    o.out_order = out_order
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
    """Frame counts of the good rays (rtb_ccd_frame).  The call runs on the
    library's own stream, which is not ordered with torch's: the device waits
    for torch's work (the zeroed counters) before it and for the frame after
    it, so the counts are complete when it returns."""
    import torch
    if counts is None:
        counts = torch.zeros(int(ccd.xdim) * int(ccd.ydim), dtype=torch.int32, device="cuda")
    if n_outside is None:
        n_outside = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    st = lib().rtb_ccd_frame(C.byref(rays.struct()), C.byref(ccd), ffi.vptr(counts), ffi.vptr(n_outside), None)
    ffi.check(st, "rtb_ccd_frame")
    torch.cuda.synchronize()
    return counts, n_outside


def reference_order(beams, n_stages: int, rays: DeviceRays):
    """The reference's Rearrange order of each beam (rtb_reference_order), on
    the library's own stream, waited for on both sides as in ccd_frame: the
    order tensor is complete when it returns."""
    import torch
    order = torch.empty(rays.n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = lib().rtb_reference_order(_beams(beams), len(beams), n_stages, C.byref(rays.struct()), ffi.vptr(order), None)
    ffi.check(st, "rtb_reference_order")
    torch.cuda.synchronize()
    return order


def specialize(surfaces, fixes=0, precision=ffi.MIXED):
    """Compile the fused kernel of `precision` specialised to this scheme's
    structure (rtb_specialize; no device needed): (status, note)."""
    arr = (ffi.Surface * len(surfaces))(*surfaces)
    note = C.create_string_buffer(4096)
    st = lib().rtb_specialize(arr, len(surfaces), fixes, precision, note, len(note))
    return st, note.value.decode()


def adjoint_specialize(surfaces, fixes=0):
    """Compile the adjoint's reverse sweep for this scheme's structure
    (rtb_adjoint_specialize; no device needed): (status, note)."""
    arr = (ffi.Surface * len(surfaces))(*surfaces)
    note = C.create_string_buffer(4096)
    st = lib().rtb_adjoint_specialize(arr, len(surfaces), fixes, note, len(note))
    return st, note.value.decode()


class Plan:
    """A batched trace (rtb_plan_*): rays generated once on the device, each
    run one CUDA graph launch of the fused kernel."""

    def __init__(self, surfaces, beams, o: ffi.TraceOpts):
        self._surf = (ffi.Surface * len(surfaces))(*surfaces)
        self._beams = _beams(beams)
        self._opts = o
        self.n_beams = len(beams)
        self.h = C.c_void_p()
        ffi.check(lib().rtb_plan_create(self._surf, len(surfaces), self._beams, len(beams), C.byref(o),
                                        C.byref(self.h)), "rtb_plan_create")

    def run(self, stream=None):
        ffi.check(lib().rtb_plan_run(self.h, stream), "rtb_plan_run")

    def result(self):
        stats = ffi.TraceStats()
        st = lib().rtb_plan_result(self.h, C.byref(stats))
        return st, stats

    def counts(self) -> np.ndarray:
        """Per-(beam, stage) counters of the last run, shape (beams, 3*surfaces+1)."""
        n = C.c_size_t(0)
        ffi.check(lib().rtb_plan_counts(self.h, None, 0, C.byref(n)), "rtb_plan_counts")
        a = np.zeros(n.value, dtype=np.uint64)
        ffi.check(lib().rtb_plan_counts(self.h, a.ctypes.data, n.value, None), "rtb_plan_counts")
        return a.reshape(self.n_beams, -1)

    def rays(self):
        i, o = ffi.Rays(), ffi.Rays()
        ffi.check(lib().rtb_plan_rays(self.h, C.byref(i), C.byref(o)), "rtb_plan_rays")
        return i, o

    def order(self, n: int):
        """The tracing order (slot -> ray index) as a device tensor of n int64,
        or None for a plan in index order."""
        import torch
        p = C.c_void_p()
        ffi.check(lib().rtb_plan_order(self.h, C.byref(p)), "rtb_plan_order")
        if not p.value:
            return None
        return torch.as_tensor(_DevArray(p.value, n, "<i4"), device="cuda").to(torch.int64) & 0xFFFFFFFF

    def autotune(self, reps=3):
        table = (ffi.TuneEntry * 16)()
        n = C.c_size_t(0)
        ffi.check(lib().rtb_plan_autotune(self.h, reps, table, 16, C.byref(n)), "rtb_plan_autotune")
        return [(t.block_size, t.rays_per_thread, t.ms) for t in table[:n.value]]

    def set_config(self, block, rpt):
        return lib().rtb_plan_set_config(self.h, block, rpt)

    def config(self):
        b, r, n = C.c_int32(), C.c_int32(), C.c_uint64()
        ffi.check(lib().rtb_plan_config(self.h, C.byref(b), C.byref(r), C.byref(n)), "rtb_plan_config")
        return b.value, r.value, n.value

    def specialized(self):
        """(True when the plan launches a kernel compiled for its scheme, why not)."""
        on = C.c_int32()
        note = C.create_string_buffer(2048)
        ffi.check(lib().rtb_plan_specialized(self.h, C.byref(on), note, len(note)), "rtb_plan_specialized")
        return bool(on.value), note.value.decode()

    def destroy(self):
        if self.h:
            lib().rtb_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Adjoint:
    """Gradients of CCD-plane positions with respect to scheme parameters
    (rtb_adjoint_*): forward(theta) -> X, Y, flag (torch device tensors),
    backward(gX, gY) -> dL/dtheta, jvp(dtheta) -> dX, dY, spot_merit()."""

    def __init__(self, surfaces, params, beams, n_rays: int, fixes: int = 0):
        import torch
        self._surf = (ffi.Surface * len(surfaces))(*surfaces)
        self._surfaces = surfaces
        self.params = list(params)
        self._params = (ffi.Param * max(1, len(self.params)))(*[ffi.Param(*p, 0) for p in self.params])
        self._beams = _beams(beams)
        self.n = n_rays
        self.h = C.c_void_p()
        ffi.check(lib().rtb_adjoint_create(self._surf, len(surfaces), self._params, len(self.params), self._beams,
                                           len(beams), n_rays, fixes, C.byref(self.h)), "rtb_adjoint_create")
        self.X = torch.empty(n_rays, dtype=torch.float64, device="cuda")
        self.Y = torch.empty(n_rays, dtype=torch.float64, device="cuda")
        self.flag = torch.empty(n_rays, dtype=torch.int8, device="cuda")

    def theta(self) -> np.ndarray:
        t = np.zeros(len(self.params))
        ffi.check(lib().rtb_adjoint_theta(self.h, t.ctypes.data), "rtb_adjoint_theta")
        return t

    @staticmethod
    def _sync():
        # inputs made by torch on its stream must be complete before the
        # library's stream reads them (the library's calls return synchronised)
        import torch
        torch.cuda.current_stream().synchronize()

    def forward(self, theta, rays: "DeviceRays"):
        self._sync()
        th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
        stats = ffi.TraceStats()
        st = lib().rtb_adjoint_forward(self.h, None if th is None else th.ctypes.data, C.byref(rays.struct()),
                                       ffi.vptr(self.X), ffi.vptr(self.Y), ffi.vptr(self.flag), C.byref(stats), None)
        return st, stats

    def backward(self, gX, gY) -> np.ndarray:
        self._sync()
        g = np.zeros(len(self.params))
        ffi.check(lib().rtb_adjoint_backward(self.h, ffi.vptr(gX), ffi.vptr(gY), g.ctypes.data, None),
                  "rtb_adjoint_backward")
        return g

    def jvp(self, dtheta):
        import torch
        d = np.ascontiguousarray(dtheta, dtype=np.float64)
        self._sync()
        dX = torch.empty(self.n, dtype=torch.float64, device="cuda")
        dY = torch.empty(self.n, dtype=torch.float64, device="cuda")
        ffi.check(lib().rtb_adjoint_jvp(self.h, d.ctypes.data, ffi.vptr(dX), ffi.vptr(dY), None), "rtb_adjoint_jvp")
        return dX, dY

    def spot_merit(self, target_x, weight: float):
        import torch
        t = np.ascontiguousarray(target_x, dtype=np.float64)
        m = C.c_double(0.0)
        gX = torch.empty(self.n, dtype=torch.float64, device="cuda")
        gY = torch.empty(self.n, dtype=torch.float64, device="cuda")
        self._sync()
        ffi.check(lib().rtb_adjoint_spot_merit(self.h, t.ctypes.data, weight, C.byref(m), ffi.vptr(gX), ffi.vptr(gY),
                                               None), "rtb_adjoint_spot_merit")
        return m.value, gX, gY

    def resolution_merit(self, lambdas, direction=(1.0, 0.0)):
        """rtb_adjoint_resolution_merit: (merit, gX, gY), the seeds on the device."""
        import torch
        lam = np.ascontiguousarray(lambdas, dtype=np.float64)
        m = C.c_double(0.0)
        gX = torch.empty(self.n, dtype=torch.float64, device="cuda")
        gY = torch.empty(self.n, dtype=torch.float64, device="cuda")
        self._sync()
        ffi.check(lib().rtb_adjoint_resolution_merit(self.h, lam.ctypes.data, float(direction[0]), float(direction[1]),
                                                     C.byref(m), ffi.vptr(gX), ffi.vptr(gY), None),
                  "rtb_adjoint_resolution_merit")
        return m.value, gX, gY

    def destroy(self):
        if self.h:
            lib().rtb_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class _DevArray:
    """A device pointer as a __cuda_array_interface__ object (zero copy)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}


def device_view(r: ffi.Rays) -> dict:
    """torch views of the non-NULL device arrays of an ffi.Rays."""
    import torch
    out = {}
    for f in FIELDS:
        p = getattr(r, f)
        if p:
            out[f] = torch.as_tensor(_DevArray(p, r.n, "<f8"), device="cuda")
    out["flag"] = torch.as_tensor(_DevArray(r.flag, r.n, "|i1"), device="cuda")
    out["lost_stage"] = torch.as_tensor(_DevArray(r.lost_stage, r.n, "|u1"), device="cuda")
    return out


class PinnedRays:
    """Host ray arrays, flags included, in page-locked memory (rtb_alocate_vector)."""

    def __init__(self, n: int):
        self.n = n
        self._ptrs = []
        for f in FIELDS:
            p = lib().rtb_alocate_vector(n)
            if not p:
                raise MemoryError("rtb_alocate_vector failed")
            self._ptrs.append(p)
            setattr(self, f, np.ctypeslib.as_array(p, shape=(n,)))
        for f, dt, v in (("flag", np.int8, 1), ("lost_stage", np.uint8, ffi.NOT_LOST)):
            p = lib().rtb_alocate_vector((n + 7) // 8)
            if not p:
                raise MemoryError("rtb_alocate_vector failed")
            self._ptrs.append(p)
            a = np.ctypeslib.as_array(p, shape=((n + 7) // 8,)).view(dt)[:n]
            a[:] = v
            setattr(self, f, a)

    def struct(self) -> ffi.Rays:
        return ffi.Rays(*(ffi.vptr(getattr(self, f)) for f in FIELDS), ffi.vptr(self.flag),
                        ffi.vptr(self.lost_stage), self.n)

    def free(self):
        for p in self._ptrs:
            lib().rtb_free_vector(p)
        self._ptrs = []
        for f in FIELDS + ("flag", "lost_stage"):
            setattr(self, f, None)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
