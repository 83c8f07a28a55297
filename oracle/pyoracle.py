"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the rt_b200 package.  The entry points
take the same arguments as the rtb_* calls of include/rtb.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from rt_b200 import ffi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build() -> None:
    """Build liboracle.so (and, where the reference sources exist, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        lib.oracle_trace.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                                     C.c_uint32, C.c_int, C.POINTER(ffi.Rays), C.POINTER(ffi.TraceStats),
                                     C.c_void_p]
        lib.oracle_trace_literal.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_uint32] + \
            [C.c_void_p] * 8 + [C.c_size_t, C.POINTER(C.c_size_t)]
        lib.oracle_generate_beams.argtypes = [C.POINTER(ffi.Beam), C.c_size_t, C.POINTER(ffi.Rays)]
        lib.oracle_reference_order.argtypes = [C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                                               C.POINTER(C.c_size_t)]
        lib.oracle_ccd_frame.argtypes = [C.POINTER(ffi.Rays), C.POINTER(ffi.CCD), C.c_void_p, C.c_void_p]
        lib.oracle_set_threads.argtypes = [C.c_int]
        lib.oracle_beam_sincos.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_philox.argtypes = [C.c_size_t, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]
        lib.oracle_spline_init.argtypes = [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_table_eval.argtypes = [C.POINTER(ffi.Table), C.c_size_t, C.c_void_p, C.c_void_p]
        lib.oracle_renormalize_count.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.c_int]
        _lib = lib
    return _lib


class HostRays:
    """SoA ray arrays in host memory."""

    FIELDS = ("X", "Y", "Z", "cX", "cY", "cZ", "lambda_")

    def __init__(self, n: int):
        self.n = n
        for f in self.FIELDS:
            setattr(self, f, np.zeros(n))
        self.flag = np.ones(n, dtype=np.int8)
        self.lost_stage = np.full(n, ffi.NOT_LOST, dtype=np.uint8)

    def struct(self) -> ffi.Rays:
        return ffi.Rays(*(ffi.vptr(getattr(self, f)) for f in self.FIELDS), ffi.vptr(self.flag),
                        ffi.vptr(self.lost_stage), self.n)

    def copy(self) -> "HostRays":
        r = HostRays(self.n)
        for f in self.FIELDS + ("flag", "lost_stage"):
            getattr(r, f)[:] = getattr(self, f)
        return r

    def take(self, idx) -> "HostRays":
        r = HostRays(len(idx))
        for f in self.FIELDS + ("flag", "lost_stage"):
            getattr(r, f)[:] = getattr(self, f)[idx]
        return r

    def state(self) -> np.ndarray:
        return np.stack([self.X, self.Y, self.Z, self.cX, self.cY, self.cZ])


def generate(beams, n: int) -> HostRays:
    rays = HostRays(n)
    arr = (ffi.Beam * len(beams))(*beams)
    st = load().oracle_generate_beams(arr, len(beams), C.byref(rays.struct()))
    ffi.check(st, "oracle_generate_beams")
    return rays


def trace(surfaces, beams, rays: HostRays, fixes: int = 0, renorm_lost: int = 1):
    """In-place per-ray trace; returns (status, stats, lost_counts[n_beams, 3*n_surf])."""
    n_s = len(surfaces)
    surf = (ffi.Surface * n_s)(*surfaces)
    barr = (ffi.Beam * len(beams))(*beams)
    stats = ffi.TraceStats()
    counts = np.zeros((len(beams), 3 * n_s), dtype=np.uint64)
    st = load().oracle_trace(surf, n_s, barr, len(beams), fixes, renorm_lost, C.byref(rays.struct()),
                             C.byref(stats), ffi.vptr(counts))
    return st, stats, counts


def count_flops(surfaces, beams, rays: HostRays, fixes: int = 0, renorm_lost: int = 1):
    """Algorithmic operation count of the reference's per-ray arithmetic over
    `rays` (not modified): (ops per surface, rays reaching each surface),
    the last entry of ops the trailing Normalize calls of lost rays."""
    L = load()
    L.oracle_count_flops.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                                     C.c_uint32, C.c_int, C.POINTER(ffi.Rays), C.c_void_p, C.c_void_p]
    n_s = len(surfaces)
    ops = np.zeros(n_s + 1, dtype=np.uint64)
    reached = np.zeros(n_s + 1, dtype=np.uint64)
    st = L.oracle_count_flops((ffi.Surface * n_s)(*surfaces), n_s, (ffi.Beam * len(beams))(*beams), len(beams),
                              fixes, renorm_lost, C.byref(rays.struct()), ffi.vptr(ops), ffi.vptr(reached))
    ffi.check(st, "oracle_count_flops")
    return ops, reached


def trace_literal(surfaces, beam, rays: HostRays, fixes: int = 0):
    """Reference-order replica for one beam covering all of `rays`; returns (status, n_good)."""
    n_s = len(surfaces)
    surf = (ffi.Surface * n_s)(*surfaces)
    ng = C.c_size_t(0)
    st = load().oracle_trace_literal(surf, n_s, C.byref(beam), fixes,
                                     *(ffi.vptr(getattr(rays, f)) for f in HostRays.FIELDS),
                                     ffi.vptr(rays.flag), rays.n, C.byref(ng))
    return st, ng.value


def reference_order(lost_stage: np.ndarray, n_stages: int):
    ls = np.ascontiguousarray(lost_stage, dtype=np.uint8)
    order = np.zeros(len(ls), dtype=np.uint32)
    ng = C.c_size_t(0)
    load().oracle_reference_order(len(ls), n_stages, ffi.vptr(ls), ffi.vptr(order), C.byref(ng))
    return order, ng.value


def ccd_frame(rays: HostRays, ccd: ffi.CCD) -> tuple[np.ndarray, int]:
    counts = np.zeros(int(ccd.xdim) * int(ccd.ydim), dtype=np.uint32)
    outside = np.zeros(1, dtype=np.uint64)
    load().oracle_ccd_frame(C.byref(rays.struct()), C.byref(ccd), ffi.vptr(counts), ffi.vptr(outside))
    return counts, int(outside[0])


def spline_init(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    y2 = np.zeros_like(x)
    ffi.check(load().oracle_spline_init(len(x), ffi.vptr(x), ffi.vptr(y), ffi.vptr(y2)), "oracle_spline_init")
    return y2


def qe_curves(cqe, rows, n_lambda: int) -> tuple[np.ndarray, np.ndarray]:
    """Scheme::ComputeQE's curves (oracle_qe_curves) for the QE surfaces of
    `cqe` (rt_b200.schemes.CQe): (lambda, qe), each n_rows x n_lambda."""
    rows = np.ascontiguousarray(np.atleast_2d(rows), dtype=np.float64)
    lam = np.zeros((rows.shape[0], n_lambda))
    qe = np.zeros_like(lam)
    L = load()
    L.oracle_qe_curves.argtypes = [C.POINTER(ffi.QeSurface), C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t,
                                   C.c_size_t, C.c_void_p, C.c_void_p]
    ffi.check(L.oracle_qe_curves(cqe.array, len(cqe), ffi.vptr(rows), rows.shape[0], rows.shape[1], n_lambda,
                                 ffi.vptr(lam), ffi.vptr(qe)), "oracle_qe_curves")
    return lam, qe


def grating_energy_distr(lam, order, blaze, alpha, gamma, gr_const, rule_start=0.0, rule_stop=1.0, energy=None):
    """grating_energy_distr (oracle_grating_energy_distr); angles in radians."""
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    e = np.ones_like(lam) if energy is None else np.array(energy, dtype=np.float64)
    L = load()
    L.oracle_grating_energy_distr.argtypes = [C.c_size_t, C.c_void_p, C.c_long] + [C.c_double] * 6 + [C.c_void_p]
    ffi.check(L.oracle_grating_energy_distr(len(lam), ffi.vptr(lam), order, blaze, alpha, gamma, gr_const,
                                            rule_start, rule_stop, ffi.vptr(e)), "oracle_grating_energy_distr")
    return e


def loss_ratios(lam, n_good: int, n_lambda: int):
    """losses_comp's (ll, ratio) for one result's wavelengths (good first)."""
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    ll, ratio = np.zeros(n_lambda), np.zeros(n_lambda)
    L = load()
    L.oracle_loss_ratios.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p, C.c_void_p]
    ffi.check(L.oracle_loss_ratios(ffi.vptr(lam), len(lam), n_good, n_lambda, ffi.vptr(ll), ffi.vptr(ratio)),
              "oracle_loss_ratios")
    return ll, ratio


def unique_lambdas(lam, n_good: int, n_lambda: int):
    """print_lambda's list of distinct good wavelengths."""
    lam = np.ascontiguousarray(lam, dtype=np.float64)
    out = np.zeros(max(1, n_good))
    n = C.c_uint64(0)
    L = load()
    L.oracle_unique_lambdas.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint64,
                                        C.POINTER(C.c_uint64)]
    ffi.check(L.oracle_unique_lambdas(ffi.vptr(lam), n_good, n_lambda, ffi.vptr(out), len(out), C.byref(n)),
              "oracle_unique_lambdas")
    return out[:n.value].copy()
