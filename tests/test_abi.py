"""The C ABI without a GPU: the library loads, exports every declared entry
point, its structs have the layout ctypes assumes, and host-only calls work.
"""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rtb.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"RTB_API\s+[\w\s\*]+?\b(rtb_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = ffi.load()
    names = declared_symbols()
    assert len(names) >= 28
    for name in names:
        assert hasattr(lib, name), name
    nm = subprocess.run(["nm", "-D", "--defined-only", ffi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (rtb_\w+)", nm))
    assert set(names) <= exported
    assert exported <= set(names), f"undeclared exports: {exported - set(names)}"


def test_struct_layouts_match_ctypes():
    structs = {"rtb_table": ffi.Table, "rtb_surface": ffi.Surface, "rtb_beam": ffi.Beam, "rtb_rays": ffi.Rays,
               "rtb_trace_opts": ffi.TraceOpts, "rtb_trace_stats": ffi.TraceStats, "rtb_ccd": ffi.CCD,
               "rtb_qe_surface": ffi.QeSurface, "rtb_scheme_beam": ffi.SchemeBeam, "rtb_param": ffi.Param,
               "rtb_tune_entry": ffi.TuneEntry}
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        src.append(f'printf("{cname} __sizeof__ %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            cf = "lambda" if fname == "lambda_" else fname
            src.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {cf}));')
    src.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        open(c, "w").write("\n".join(src))
        exe = os.path.join(d, "layout")
        subprocess.run(["gcc", c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in out:
        if not line:
            continue
        cname, field, val = line.split()
        py = structs[cname]
        got = C.sizeof(py) if field == "__sizeof__" else getattr(py, field).offset
        assert got == int(val), (cname, field, got, val)


def test_spline_init_matches_oracle_and_scipy():
    from scipy.interpolate import CubicSpline
    from rt_b200 import schemes as S
    for x, y in (S.glass_table(), S.qe_table()):
        y2 = E.spline_init(x, y)
        assert np.array_equal(y2.view(np.uint64), O.spline_init(x, y).view(np.uint64))
        ref = CubicSpline(x, y, bc_type="natural")(x, 2)
        np.testing.assert_allclose(y2, ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())


def test_spline_init_rejects_short_tables():
    x = np.array([0.1, 0.2, 0.3])
    assert E.lib().rtb_spline_init(3, ffi.vptr(x), ffi.vptr(x), ffi.vptr(np.zeros(3))) == ffi.BAD_VALUE


def test_calls_fail_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert E.lib().rtb_init() == ffi.INIT_FAILED
    n = 4
    a = [np.zeros(n) for _ in range(6)]
    nb = C.c_size_t(0)
    st = E.lib().rtb_surface_intersection(0, ffi.dptr(np.zeros(16)), C.c_size_t(n), *(ffi.dptr(x) for x in a),
                                          C.byref(nb), ffi.vptr(np.ones(n, dtype=np.int8)))
    assert st == ffi.INIT_FAILED
