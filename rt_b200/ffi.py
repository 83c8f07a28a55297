"""ctypes mirror of include/rtb.h and the loader of librtb200.so.

The structures here are byte-for-byte the C structs of include/rtb.h; the
Python layer only marshals arguments.  All computation happens in the CUDA
library; `load()` raises if it is missing, there is no Python fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtb200.so")

# status codes (rtb.h)
OK, INIT_FAILED, BAD_ALLOC, FAILED, BAD_VALUE, NO_INTERSECTIONS, NO_GOOD_RAYS, OUT_OF_RANGE = range(8)
STATUS_NAMES = {
    OK: "OK", INIT_FAILED: "INIT_FAILED", BAD_ALLOC: "BAD_ALLOC", FAILED: "FAILED",
    BAD_VALUE: "BAD_VALUE", NO_INTERSECTIONS: "NO_INTERSECTIONS", NO_GOOD_RAYS: "NO_GOOD_RAYS",
    OUT_OF_RANGE: "OUT_OF_RANGE",
}

# enumerations (common-lib/surface.h:130-132,241)
PLANE, CONIC, TORIC, AUX_CLASS = range(4)
MIRROR, LENS, GRATING, STOP, SHADE, DETECTOR, AUX_TYPE = range(7)
CIRCLE, RECTANGLE = range(2)
REFLECTIVE, TRANSPARENT = range(2)
ENGINE_PER_SURFACE, ENGINE_FUSED = range(2)
FP64, MIXED, MIXED32 = range(3)
FIX_TORIC_SIGN = 1
FIX_TORIC_STEP = 2
FIX_ASPHERE_ROOT = 4
ORDER_COHERENT, ORDER_INDEX = 0, 1
OUT_INDEX, OUT_SLOT = 0, 1

MAX_POLY = 10
MAX_PARAMS = 16
MAX_SURFACES = 32
MAX_GRATINGS = 8
MAX_KNOTS = 1024
NOT_LOST = 0xFF


class Table(C.Structure):
    _fields_ = [("n", C.c_size_t), ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
                ("y2", C.POINTER(C.c_double))]


class Surface(C.Structure):
    _fields_ = [("cls", C.c_int32), ("type", C.c_int32), ("shape", C.c_int32), ("grating_type", C.c_int32),
                ("order", C.c_int64), ("gr_const", C.c_double), ("params", C.c_double * MAX_PARAMS),
                ("size", C.c_double * 2), ("center", C.c_double * 2), ("distance", C.c_double * 3),
                ("angles_deg", C.c_double * 3), ("n1", Table), ("n2", Table)]


class Beam(C.Structure):
    _fields_ = [("first_ray", C.c_uint64), ("n_rays", C.c_uint64), ("orders", C.c_int64 * MAX_GRATINGS),
                ("n_orders", C.c_int32), ("shape", C.c_int32), ("disk", C.c_double * 3),
                ("center", C.c_double * 3), ("range", C.c_double * 2), ("n_lambda", C.c_uint64),
                ("field", C.c_double * 2), ("seed", C.c_uint64)]


class Rays(C.Structure):
    _fields_ = [("X", C.c_void_p), ("Y", C.c_void_p), ("Z", C.c_void_p), ("cX", C.c_void_p),
                ("cY", C.c_void_p), ("cZ", C.c_void_p), ("lambda_", C.c_void_p), ("flag", C.c_void_p),
                ("lost_stage", C.c_void_p), ("n", C.c_size_t)]


class CCD(C.Structure):
    _fields_ = [("xsize", C.c_double), ("ysize", C.c_double), ("xdim", C.c_uint64), ("ydim", C.c_uint64),
                ("xpix", C.c_double), ("ypix", C.c_double)]


class TraceOpts(C.Structure):
    _fields_ = [("engine", C.c_int32), ("precision", C.c_int32), ("fixes", C.c_uint32),
                ("renormalize_lost", C.c_int32), ("block_size", C.c_int32), ("rays_per_thread", C.c_int32),
                ("state_out", C.c_int32), ("ray_order", C.c_int32), ("ccd", C.POINTER(CCD)),
                ("counts", C.c_void_p), ("n_outside", C.c_void_p), ("out_order", C.c_int32),
                ("reserved", C.c_int32)]


class TraceStats(C.Structure):
    _fields_ = [("ray_surfaces", C.c_uint64), ("n_good", C.c_uint64), ("failed_beam", C.c_int32),
                ("failed_stage", C.c_int32)]


class Param(C.Structure):
    _fields_ = [("surface", C.c_int32), ("kind", C.c_int32), ("index", C.c_int32), ("reserved", C.c_int32)]


PARAM_CURVATURE, PARAM_CONIC, PARAM_POLY, PARAM_TORIC_CR, PARAM_DISTANCE, PARAM_ANGLE, PARAM_GROOVE_DENSITY = range(7)
ADJ_MAX_PARAMS = 64


class SchemeBeam(C.Structure):
    _fields_ = [("type", C.c_int32), ("shape", C.c_int32), ("profile", C.c_int32), ("range_distr", C.c_int32),
                ("params", C.c_double * 6), ("n_params", C.c_int32), ("reserved", C.c_int32),
                ("center", C.c_double * 3), ("n_lambda", C.c_uint64)]


class QeSurface(C.Structure):
    _fields_ = [("type", C.c_int32), ("reserved", C.c_int32), ("qe", Table), ("order", C.c_int64),
                ("gr_const", C.c_double), ("alpha_deg", C.c_double), ("gamma_deg", C.c_double),
                ("blaze_deg", C.c_double), ("rule_start", C.c_double), ("rule_stop", C.c_double)]


class TuneEntry(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("rays_per_thread", C.c_int32), ("ms", C.c_double)]


def dptr(a: np.ndarray) -> C.POINTER(C.c_double):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def vptr(a) -> C.c_void_p:
    """Address of a numpy array (host) or of a torch tensor (device)."""
    if a is None:
        return C.c_void_p(0)
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())


class TableHolder:
    """Keeps the numpy arrays of an rtb_table alive."""

    def __init__(self, x=None, y=None, value=None):
        if value is not None:
            self.x = np.zeros(1)
            self.y = np.array([float(value)])
            self.y2 = np.zeros(1)
        else:
            self.x = np.ascontiguousarray(x, dtype=np.float64)
            self.y = np.ascontiguousarray(y, dtype=np.float64)
            self.y2 = np.zeros_like(self.x)
        self.table = Table(len(self.x), dptr(self.x), dptr(self.y), dptr(self.y2))

    @property
    def single(self) -> bool:
        return len(self.x) == 1


_lib = None


def load() -> C.CDLL:
    """Load librtb200.so (raises if the CUDA library was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python __graft_entry__.py build` (or build())")
        _lib = C.CDLL(LIB_PATH)
    return _lib


def check(status: int, what: str = "rtb call") -> int:
    if status != OK:
        raise RuntimeError(f"{what} failed: {STATUS_NAMES.get(status, status)}")
    return status
