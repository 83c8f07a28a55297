"""Scheme-specialised fused kernels (jit.cpp) without a GPU: rtb_specialize
compiles the fused mixed and FP64 kernels for the structure of every
benchmark and coverage scheme with NVRTC."""
import ctypes as C

import pytest

import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

SCHEMES = {
    "c0": S.littrow_free,
    "c0_asphere": S.c0_asphere_camera,
    "c4": S.littrow_free_asphere,
    "c1": S.echelle,
    "mirrors": lambda: S.coverage_schemes()["mirrors"],
    "lenses": lambda: S.coverage_schemes()["lenses"],
    "gratings": lambda: S.coverage_schemes()["gratings"],
}


def _nvrtc_present():
    try:
        C.CDLL("libnvrtc.so.12")
        return True
    except OSError:
        try:
            C.CDLL("/usr/local/cuda/lib64/libnvrtc.so.12")
            return True
        except OSError:
            return False


@pytest.mark.skipif(not _nvrtc_present(), reason="libnvrtc not present")
@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.FP64])
@pytest.mark.parametrize("name", sorted(SCHEMES))
def test_specialised_kernel_compiles(name, precision):
    cs = S.to_c(SCHEMES[name](), O.spline_init)
    st, note = E.specialize(list(cs.surfaces), ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP, precision)
    assert st == ffi.OK, note
    assert note == ""


def test_specialize_rejects_bad_requests():
    st, _ = E.specialize([], 0)
    assert st == ffi.BAD_VALUE
    cs = S.to_c(S.littrow_free(), O.spline_init)
    st, _ = E.specialize(list(cs.surfaces), 0, 7)
    assert st == ffi.BAD_VALUE
