"""rt_trace, the reference's ray-tracing program on the B200 engine (GPU tests).

Runs rt_b200/bin/rt_trace on scheme files and checks its .dat results bit
for bit against the CPU oracle's literal replica of Scheme::run (which writes
rays in the order the reference's Rearrange calls leave them, pinned to the
reference's own Beam::Save output by tests/test_oracle_pins.py).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import pyoracle as O
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RT_TRACE = os.path.join(ROOT, "rt_b200", "bin", "rt_trace")
SEED = 1234


def read_dat(path):
    L = ffi.load()
    n, ng, nl = C.c_uint64(), C.c_uint64(), C.c_uint64()
    assert L.rtb_read_dat_header(path.encode(), C.byref(n), C.byref(ng), C.byref(nl)) == ffi.OK
    r = O.HostRays(n.value)
    L.rtb_read_dat.argtypes = [C.c_char_p, C.POINTER(ffi.Rays)]
    assert L.rtb_read_dat(path.encode(), C.byref(r.struct())) == ffi.OK
    return r, ng.value, nl.value


def run(tmp_path, xml, *extra):
    out = subprocess.run([RT_TRACE, xml, "rt_files.txt", "log.txt", "--seed", str(SEED), *extra], cwd=str(tmp_path),
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr + out.stdout
    return [ln.strip() for ln in open(tmp_path / "rt_files.txt") if ln.strip()]


def oracle_range(specs, n_per, n_lambda, radius, w, seed, orders=()):
    beam = S.make_beam(0, n_per, n_lambda, radius, w, seed, orders=orders)
    rays = O.generate([beam], beam.n_rays)
    inp = rays.copy()
    cs = S.to_c(specs, O.spline_init)
    st, ng = O.trace_literal(cs.surfaces, beam, rays)
    return inp, rays, st, ng


def assert_same(dat, ora_rays, ng_expected):
    r, ng, _ = dat
    assert ng == ng_expected
    for f in O.HostRays.FIELDS:
        a, b = getattr(r, f), getattr(ora_rays, f)
        same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
        assert same.all(), f


def test_single_range_scheme_file(tmp_path):
    """C0's committed scheme file: one composite range of 5 wavelengths."""
    xml = os.path.join(ROOT, "rt_b200", "data", "c0_littrow_free.xml")
    files = run(tmp_path, xml)
    assert files == ["c0.dat"]
    inp, ora, st, ng = oracle_range(S.littrow_free(), 20000, 5, S.C0_RADIUS, S.C0_LAMBDA, SEED)
    assert st == ffi.OK
    dat_in = read_dat(str(tmp_path / "c0_input_beam.dat"))
    assert_same(dat_in, inp, inp.n)
    assert_same(read_dat(str(tmp_path / "c0.dat")), ora, ng)


def test_range_file_with_orders(tmp_path):
    """C1 with a range file of three echelle orders: one result per range,
    named <root>_range_(w1-w2).dat as the reference names them, orders taken
    from the range rows."""
    ranges = [[0.38, 0.9, m, 1] for m in (33, 45, 58)]
    xml = str(tmp_path / "c1_small.xml")
    S.write_xml(xml, S.echelle(), "C1 small", "c1s", 300, S.C1_RADIUS, ranges, n_lambda=S.C1_NLAMBDA)
    files = run(tmp_path, xml)
    assert len(files) == 3
    for r, (row, fn) in enumerate(zip(ranges, files)):
        assert fn == "c1s_range_(0.38-0.9).dat"
        _, ora, st, ng = oracle_range(S.echelle(), 300, S.C1_NLAMBDA, S.C1_RADIUS, row[:2], SEED + r,
                                      orders=row[2:])
        assert st == ffi.OK
    # every range writes the same file name (as in the reference): the last one remains
    assert_same(read_dat(str(tmp_path / files[-1])), ora, ng)


def test_mixed_precision_runner(tmp_path):
    xml = os.path.join(ROOT, "rt_b200", "data", "c0_littrow_free.xml")
    run(tmp_path, xml, "--precision", "mixed")
    _, ora, st, ng = oracle_range(S.littrow_free(), 20000, 5, S.C0_RADIUS, S.C0_LAMBDA, SEED)
    r, ng_m, _ = read_dat(str(tmp_path / "c0.dat"))
    assert abs(ng_m - ng) <= 2
    # good rays of both, compared by position in the good prefix is not meaningful
    # if a flag differs; compare the CCD positions as sets of the common good rays
    a = np.sort(np.round(r.X[:ng_m], 6))
    b = np.sort(np.round(ora.X[:ng], 6))
    k = min(len(a), len(b))
    assert np.abs(a[:k] - b[:k]).max() < 1e-4


RT_CCD = os.path.join(ROOT, "rt_b200", "bin", "rt_ccd_frame")


def test_ccd_frame_program(tmp_path):
    """rt_trace then rt_ccd_frame on C0: the FITS image equals the image the
    CPU oracle's ccd_coordinates / compute_ccd_image make from the same .dat
    file, QE block and spectrum (FP64 sums in a different order: 1e-12)."""
    xml = os.path.join(ROOT, "rt_b200", "data", "c0_littrow_free.xml")
    files = run(tmp_path, xml)
    (tmp_path / "rt_list.txt").write_text("".join(f + "\n" for f in files))
    qx, qy = S.qe_table()
    with open(tmp_path / "qe.bin", "wb") as f:
        f.write(np.array([len(qx)], dtype=np.uint64).tobytes() + qx.tobytes() + qy.tobytes())
    sx = np.linspace(0.3, 0.9, 13)
    S.write_table(str(tmp_path / "spec.txt"), sx, 1.0 + 0.5 * sx)
    c = S.C0_CCD
    (tmp_path / "ccd.txt").write_text(f"# CCD\n{c['xsize']} {c['ysize']}\n{c['xdim']} {c['ydim']}\n"
                                      f"{c['xpix']} {c['ypix']}\n")
    out = subprocess.run([RT_CCD, "rt_list.txt", "qe.bin", "spec.txt", "ccd.txt", "frame.fits"], cwd=str(tmp_path),
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr + out.stdout
    raw = open(tmp_path / "frame.fits", "rb").read()
    img = np.frombuffer(raw[2880:2880 + 8 * c["xdim"] * c["ydim"]], dtype=">f8").reshape(c["ydim"], c["xdim"])
    # the oracle on the same rays
    r, ng, _ = read_dat(str(tmp_path / files[0]))
    Lo = O.load()
    cx, cy = np.zeros(ng, dtype=np.uint32), np.zeros(ng, dtype=np.uint32)
    Lo.oracle_ccd_coordinates(C.c_size_t(ng), ffi.dptr(r.X), ffi.dptr(r.Y), C.c_double(c["xsize"]),
                              C.c_double(c["ysize"]), C.c_double(c["xpix"]), C.c_double(c["ypix"]),
                              ffi.vptr(cx), ffi.vptr(cy))
    qt = ffi.TableHolder(x=qx, y=qy)
    qt.y2[:] = O.spline_init(qt.x, qt.y)
    st = ffi.TableHolder(x=sx, y=1.0 + 0.5 * sx)
    st.y2[:] = O.spline_init(st.x, st.y)
    ref = np.zeros(c["xdim"] * c["ydim"])
    nout = C.c_uint64(0)
    assert Lo.oracle_compute_ccd_image(C.c_size_t(ng), ffi.vptr(cx), ffi.vptr(cy), ffi.dptr(r.lambda_),
                                       C.byref(qt.table), C.byref(st.table), C.c_size_t(c["xdim"]),
                                       C.c_size_t(c["ydim"]), C.c_double(c["xpix"]), C.c_double(c["ypix"]),
                                       ffi.dptr(ref), C.byref(nout)) == ffi.OK
    ref = ref.reshape(c["ydim"], c["xdim"])
    assert ref.sum() > 0
    assert np.allclose(img, ref, rtol=1e-12, atol=0)
