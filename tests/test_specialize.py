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
@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32, ffi.FP64])
@pytest.mark.parametrize("name", sorted(SCHEMES))
def test_specialised_kernel_compiles(name, precision):
    cs = S.to_c(SCHEMES[name](), O.spline_init)
    st, note = E.specialize(list(cs.surfaces), ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP, precision)
    assert st == ffi.OK, note
    assert note == ""


@pytest.mark.skipif(not _nvrtc_present(), reason="libnvrtc not present")
@pytest.mark.parametrize("name", sorted(SCHEMES))
def test_adjoint_reverse_sweep_compiles(name):
    """The adjoint's reverse sweep compiled for each scheme's structure
    (rtb_adjoint_specialize, adjoint_rev.cuh with one AdjShape per surface)."""
    cs = S.to_c(SCHEMES[name](), O.spline_init)
    st, note = E.adjoint_specialize(list(cs.surfaces), ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP)
    assert st == ffi.OK, note
    assert note == ""


def test_specialize_rejects_bad_requests():
    st, _ = E.specialize([], 0)
    assert st == ffi.BAD_VALUE
    cs = S.to_c(S.littrow_free(), O.spline_init)
    st, _ = E.specialize(list(cs.surfaces), 0, 7)
    assert st == ffi.BAD_VALUE


def _specialize_in_subprocess(cache_dir):
    """rtb_specialize of C1's structure in a fresh process with the disk
    cache at cache_dir: (status, seconds)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys, time; sys.path[:0] = [%r, %r]\n"
            "import pyoracle as O\n"
            "from rt_b200 import engine as E, ffi, schemes as S\n"
            "cs = S.to_c(S.echelle(), O.spline_init)\n"
            "t = time.perf_counter(); st, note = E.specialize(list(cs.surfaces), 3, ffi.MIXED)\n"
            "print(st, time.perf_counter() - t)\n") % (root, os.path.join(root, "oracle"))
    env = dict(os.environ, RTB_JIT_CACHE=str(cache_dir))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    st, dt = out.stdout.split()
    return int(st), float(dt)


@pytest.mark.skipif(not _nvrtc_present(), reason="libnvrtc not present")
def test_jit_disk_cache(tmp_path):
    """With RTB_JIT_CACHE set, the first process compiles and stores the
    kernel, a second one loads it instead of compiling; a file whose key does
    not match is ignored and replaced."""
    st, t_compile = _specialize_in_subprocess(tmp_path)
    assert st == ffi.OK
    files = list(tmp_path.glob("rtb-*.cubin"))
    assert len(files) == 1 and not list(tmp_path.glob("*.tmp.*"))
    st, t_cached = _specialize_in_subprocess(tmp_path)
    assert st == ffi.OK and t_cached < t_compile and len(list(tmp_path.glob("rtb-*.cubin"))) == 1
    # damage the stored key: the next process compiles again and rewrites it
    data = bytearray(files[0].read_bytes())
    data[20] ^= 0xFF
    files[0].write_bytes(bytes(data))
    st, _ = _specialize_in_subprocess(tmp_path)
    assert st == ffi.OK and files[0].read_bytes() != bytes(data)


@pytest.mark.skipif(not _nvrtc_present(), reason="libnvrtc not present")
@pytest.mark.parametrize("mode", ["values", "structure"])
def test_kernels_are_shared_by_what_they_bake(tmp_path, mode):
    """By default a kernel bakes in its scheme's surface constants: C0 with
    another collimator curvature and camera distance compiles to a kernel of
    its own.  With RTB_SPECIALIZE=structure only the structure is fixed: the
    two compile to the same kernel (one cache file), C0 with an asphere
    camera to another."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path[:0] = [%r, %r]\n"
            "import pyoracle as O\n"
            "from rt_b200 import engine as E, ffi, schemes as S\n"
            "a = S.littrow_free()\n"
            "b = S.littrow_free(); b[0].params = (-1 / 750.0, -1.0, 0); b[2].distance = (1.0, 2.0, 3.0)\n"
            "c = S.c0_asphere_camera()\n"
            "for specs in (a, b, c):\n"
            "    st, note = E.specialize(list(S.to_c(specs, O.spline_init).surfaces), 0, ffi.FP64)\n"
            "    assert st == ffi.OK, note\n"
            "    print(len([f for f in __import__('os').listdir(%r) if f.endswith('.cubin')]))\n"
            ) % (root, os.path.join(root, "oracle"), str(tmp_path))
    env = dict(os.environ, RTB_JIT_CACHE=str(tmp_path))
    if mode == "structure":
        env["RTB_SPECIALIZE"] = "structure"
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == (["1", "2", "3"] if mode == "values" else ["1", "1", "2"])
