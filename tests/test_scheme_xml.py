"""Scheme files (rtb_scheme_load): the reference's XML format read by the
library without Mini-XML (no GPU needed).

* Writing a scheme with schemes.write_xml and loading it back gives the same
  rtb_surface values (tables included), beam and ranges.
* The committed scheme files in rt_b200/data are the benchmark schemes.
* Malformed files fail with the Scheme::SchemeError the reference throws
  (common-lib/scheme.h:25-27).
"""
import os

import numpy as np
import pytest

import pyoracle as O
from rt_b200 import ffi, schemes as S

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(os.path.dirname(HERE), "rt_b200", "data")

FILE_OPEN, PARSE, BAD_ATTR, NAN_ATTR = 0, 1, 3, 4
NO_SCHEME, NO_BEAM, NO_SURFACE, NO_RANGE_FILE, BAD_RANGE = 6, 7, 8, 10, 11


def table_values(t):
    if t.n == 1:
        return [t.y[0]]
    n = t.n
    return [t.x[i] for i in range(n)] + [t.y[i] for i in range(n)] + [t.y2[i] for i in range(n)]


def assert_same_surfaces(loaded, specs):
    ref = S.to_c(specs, O.spline_init).surfaces
    assert len(loaded) == len(ref)
    for a, b in zip(loaded, ref):
        for f in ("cls", "type", "shape", "order"):
            assert getattr(a, f) == getattr(b, f), f
        if b.type == ffi.GRATING:
            assert a.grating_type == b.grating_type and a.gr_const == b.gr_const
        if b.cls != ffi.AUX_CLASS:
            assert list(a.params) == list(b.params)
            assert list(a.size)[:1] == list(b.size)[:1] and list(a.center) == list(b.center)
        assert list(a.distance) == list(b.distance) and list(a.angles_deg) == list(b.angles_deg)
        if b.type in (ffi.LENS, ffi.GRATING):
            for t in ("n1", "n2"):
                va, vb = table_values(getattr(a, t)), table_values(getattr(b, t))
                assert len(va) == len(vb)
                assert np.allclose(va, vb, rtol=0, atol=1e-15), t


CASES = {
    "c0": (S.littrow_free, [[0.4, 0.7]], 5),
    "c1": (S.echelle, [[0.38, 0.9, m, 1] for m in S.C1_ORDERS], 64),
    "c4": (S.littrow_free_asphere, [[0.4, 0.7]], 64),
    "mirrors": (lambda: S.coverage_schemes()["mirrors"], [[0.4, 0.8]], 0),
    "lenses": (lambda: S.coverage_schemes()["lenses"], [[0.4, 0.8]], 0),
    "gratings": (lambda: S.coverage_schemes()["gratings"], [[0.4, 0.8, 1, -1, 1, 1, 1, 2]] * 2, 0),
}


@pytest.mark.parametrize("name", list(CASES))
def test_write_then_load_round_trip(name, tmp_path):
    make, ranges, nl = CASES[name]
    specs = make()
    path = str(tmp_path / f"{name}.xml")
    S.write_xml(path, specs, f"scheme {name}", f"res_{name}", 1000, 12.5, ranges, n_lambda=nl)
    cwd = os.getcwd()
    os.chdir(str(tmp_path))  # table and range files are named relative to the working directory
    try:
        sc = S.LoadedScheme(path)
    finally:
        os.chdir(cwd)
    assert sc.status == ffi.OK, sc.scheme_error
    assert sc.name == f"scheme {name}" and sc.result_file == f"res_{name}" and sc.log_file == ""
    assert_same_surfaces(sc.surfaces, specs)
    assert sc.comments == [s.comment for s in specs]
    assert np.array_equal(sc.ranges, np.array(ranges, dtype=float))
    b = sc.beam
    assert (b.type, b.shape, b.profile, b.range_distr) == (0, ffi.CIRCLE, 0, 1)
    assert list(b.params[:b.n_params]) == [1000.0, 0.0, 12.5] and b.n_lambda == nl


def test_committed_scheme_files_are_the_benchmark_schemes():
    for fn, make, nr in (("c0_littrow_free.xml", S.littrow_free, 1), ("c1_echelle.xml", S.echelle, 31),
                         ("c4_littrow_free_flattener.xml", S.littrow_free_asphere, 1)):
        sc = S.LoadedScheme(os.path.join(DATA, fn))  # tables found beside the scheme file
        assert sc.status == ffi.OK, (fn, sc.scheme_error)
        assert_same_surfaces(sc.surfaces, make())
        assert sc.ranges.shape[0] == nr


def write(tmp_path, body, name="s.xml"):
    p = tmp_path / name
    p.write_text(body)
    return str(p)


GOOD_SURFACE = """<surface><class>PLANE</class><type>MIRROR</type><shape>CIRC</shape><params>0 0 0</params>
<size>10</size><center>0 0</center><distance>0 0 10</distance><angles>0 0 0</angles></surface>"""
GOOD_BEAM = """<beam><type>PARALLEL</type><shape>CIRC</shape><profile>RANDOM</profile>
<range_distr>UNIFORM</range_distr><params>100 0 5</params><center>0 0 0</center><range>0.4 0.7</range></beam>"""
GENERAL = "<general><name>t</name><result_file>r</result_file></general>"


@pytest.mark.parametrize("body,err", [
    (None, FILE_OPEN),
    ("<scheme><general><name>t</name></scheme>", PARSE),
    ("<scheme>" + GOOD_SURFACE + GOOD_BEAM + "</scheme>", NO_SCHEME),
    ("<scheme>" + GENERAL + GOOD_BEAM + "</scheme>", NO_SURFACE),
    ("<scheme>" + GENERAL + GOOD_SURFACE + "</scheme>", NO_BEAM),
    ("<scheme>" + GENERAL + GOOD_SURFACE.replace("PLANE", "SPHERE") + GOOD_BEAM + "</scheme>", BAD_ATTR),
    ("<scheme>" + GENERAL + GOOD_SURFACE.replace("<size>10</size>", "<size>  </size>") + GOOD_BEAM + "</scheme>",
     BAD_ATTR),
    ("<scheme>" + GENERAL + GOOD_SURFACE.replace("<angles>0 0 0</angles>", "") + GOOD_BEAM + "</scheme>", PARSE),
    ("<scheme>" + GENERAL + GOOD_SURFACE + GOOD_BEAM.replace("0.4 0.7", "0.7 0.4") + "</scheme>", BAD_RANGE),
    ("<scheme>" + GENERAL + GOOD_SURFACE + GOOD_BEAM.replace("0.4 0.7", "missing_ranges.txt") + "</scheme>",
     NO_RANGE_FILE),
])
def test_malformed_files_fail_like_the_reference(tmp_path, body, err):
    path = str(tmp_path / "absent.xml") if body is None else write(tmp_path, body)
    sc = S.LoadedScheme(path)
    assert sc.status == ffi.BAD_VALUE and sc.scheme_error == err


def test_values_and_names(tmp_path):
    """Values are element texts with spaces and tabs trimmed; words are
    upper-cased (class, type, shape), names kept; an n1 that is not purely a
    number is a table file; comments and entities are understood."""
    (tmp_path / "glass.txt").write_text("# x y\n0.3 1.5\n0.5 1.49\n0.7 1.48\n0.9 1.47\n")
    body = ("<?xml version='1.0'?><!-- a scheme --><scheme>" + GENERAL.replace("<name>t</name>", "<name> My &amp; scheme\t</name>") +
            "<surface><class> conic </class><type>lens</type><shape>circle</shape><params>0.01 0 0</params>"
            "<size>20</size><center>0 0</center><distance>0 0 50</distance><angles>0 1.5 0</angles>"
            "<n1>1.0</n1><n2>glass.txt</n2><comment>front</comment></surface>"
            + GOOD_BEAM.replace("</beam>", "<nlambda>16</nlambda></beam>") + "</scheme>")
    cwd = os.getcwd()
    os.chdir(str(tmp_path))
    try:
        sc = S.LoadedScheme(write(tmp_path, body))
    finally:
        os.chdir(cwd)
    assert sc.status == ffi.OK, sc.scheme_error
    assert sc.name == "My & scheme"
    s = sc.surfaces[0]
    assert (s.cls, s.type, s.shape) == (ffi.CONIC, ffi.LENS, ffi.CIRCLE)
    assert s.n1.n == 1 and s.n1.y[0] == 1.0 and s.n2.n == 4
    assert [s.n2.x[i] for i in range(4)] == [0.3, 0.5, 0.7, 0.9]
    y2 = O.spline_init(np.array([0.3, 0.5, 0.7, 0.9]), np.array([1.5, 1.49, 1.48, 1.47]))
    assert np.allclose([s.n2.y2[i] for i in range(4)], y2, rtol=0, atol=1e-15)
    assert list(s.angles_deg) == [0.0, 1.5, 0.0] and sc.comments == ["front"] and sc.beam.n_lambda == 16


def test_fits_writer(tmp_path):
    """rtb_write_fits: a FITS primary image as ccd_frame writes it (BITPIX -64,
    big-endian doubles, 2880-byte blocks, string keywords)."""
    import ctypes as C
    L = ffi.load()
    L.rtb_write_fits.argtypes = [C.c_char_p, C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_char_p),
                                 C.POINTER(C.c_char_p), C.c_size_t]
    img = np.arange(7 * 5, dtype=np.float64).reshape(5, 7) * 0.25 - 3.0
    keys = (C.c_char_p * 2)(b"RT_LIST", b"CCDINFO")
    vals = (C.c_char_p * 2)(b"rt_files.txt", b"it's ccd.txt")
    path = str(tmp_path / "f.fits")
    assert L.rtb_write_fits(path.encode(), img.ctypes.data, 7, 5, keys, vals, 2) == ffi.OK
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    cards = [raw[i:i + 80].decode() for i in range(0, 2880, 80)]
    kv = {c[:8].strip(): c[10:].split("/")[0].strip() for c in cards if c[8:10] == "= "}
    assert cards[0].startswith("SIMPLE  =") and kv["SIMPLE"] == "T"
    assert kv["BITPIX"] == "-64" and kv["NAXIS"] == "2" and kv["NAXIS1"] == "7" and kv["NAXIS2"] == "5"
    assert kv["RT_LIST"].startswith("'rt_files.txt") and kv["CCDINFO"].startswith("'it''s ccd.txt")
    end = [i for i, c in enumerate(cards) if c.startswith("END")][0]
    assert all(c == " " * 80 for c in cards[end + 1:])
    data = np.frombuffer(raw[2880:2880 + 8 * 35], dtype=">f8").reshape(5, 7)
    assert np.array_equal(data, img)
    assert raw[2880 + 8 * 35:] == b"\0" * (len(raw) - 2880 - 8 * 35)
