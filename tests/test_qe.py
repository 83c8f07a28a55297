"""Throughput curves (Scheme::ComputeQE, common-lib/scheme.cpp:1123-1338)
without a GPU: the oracle against the reference's own host classes and
against fixtures of the reference's CUDA engine, the scheme reader's QE
attributes and error codes, and the QE file writer.
"""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle as O
import qe_cases as Q
import refharness as H
from rt_b200 import ffi, schemes as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "qe_refgpu.npz")
CASES = Q.cases()


def bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


def assert_curves_close(got, ref, tol=1e-12):
    """Curves from different implementations of sin, cos and asin: NaN in
    the same places, every other value within tol of the block's largest."""
    got, ref = np.atleast_2d(got), np.atleast_2d(ref)
    for g, r in zip(got, ref):
        nan = np.isnan(r)
        assert np.array_equal(np.isnan(g), nan)
        if nan.all():
            continue
        scale = np.abs(r[~nan]).max()
        err = np.abs(g[~nan] - r[~nan]).max()
        assert err <= tol * scale, err / scale


@pytest.mark.skipif(H.harness("cpu") is None, reason="reference harness not built")
@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_matches_reference_host_classes(case):
    """The reference's Surface/Grating::ApplyQE with SetRuleParams and
    ComputeQE's loop (harness_cpu, over the oracle's engine functions) and the
    oracle's restatement of that loop give the same bits."""
    specs, rows, n_lambda = CASES[case]
    cq = S.qe_surfaces(specs, O.spline_init)
    lam, qe = O.qe_curves(cq, rows, n_lambda)
    rc, blocks = H.run_qe("cpu", specs, rows, n_lambda)
    assert rc == 0
    assert len(blocks) == len(rows)
    for r, (bl, bq) in enumerate(blocks):
        assert bits_equal(bl, lam[r])
        assert bits_equal(bq, qe[r])
    if case == "evanescent":
        assert np.isnan(qe[0, -1]) and np.isfinite(qe[0, 0])
    else:
        assert np.all(np.isfinite(qe)) and np.all(qe >= 0) and np.all(qe <= 1)


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_matches_reference_cuda_engine_fixture(case):
    """The oracle against the reference's cuda_engine (surface_QE and
    grating_energy_distr kernels on a B200, single-value QE curves): the
    blaze function's sin, cos and asin differ from the host's in the last
    bits."""
    specs, rows, n_lambda = CASES[case]
    g = np.load(GOLDEN)
    cq = S.qe_surfaces(Q.scalar_qe(specs), O.spline_init)
    lam, qe = O.qe_curves(cq, rows, n_lambda)
    assert bits_equal(lam, g[case + "_lambda"])
    assert_curves_close(qe, g[case + "_qe"], Q.tolerance(case))


def test_oracle_errors_follow_the_reference():
    rows, n = [[0.4, 0.7]], 33
    bad_rule = [Q.grating(1, 1.0 / 0.6, 10.0, 0.0, 9.5, rule=(0.6, 0.3))]
    cq = S.qe_surfaces(bad_rule, O.spline_init)
    with pytest.raises(RuntimeError):
        O.qe_curves(cq, rows, n)
    x, y = S.qe_table()
    short = [S.SurfaceSpec(ffi.PLANE, ffi.MIRROR, qe=(x, y))]
    cq = S.qe_surfaces(short, O.spline_init)
    with pytest.raises(RuntimeError, match="OUT_OF_RANGE"):
        O.qe_curves(cq, [[0.4, 0.8]], n)
    if H.harness("cpu") is not None:
        assert H.run_qe("cpu", bad_rule, rows, n)[0] == 4       # Grating::BadRuleParams
        assert H.run_qe("cpu", short, [[0.4, 0.8]], n)[0] == 7  # TabulatedFunction::OutOfRange


def write_scheme(tmp_path, specs, ranges=((0.4, 0.7),), name="s.xml"):
    path = str(tmp_path / name)
    S.write_xml(path, specs, "qe test", "qe", 100, 10.0, [list(r) for r in ranges], n_lambda=5)
    return path


def test_scheme_qe_attributes(tmp_path):
    specs = S.littrow_free()
    specs[1].rule_params = (0.2,)
    sc = S.LoadedScheme(write_scheme(tmp_path, specs))
    assert sc.status == ffi.OK and sc.qe_status == ffi.OK and sc.qe_error == -1
    assert sc.n_qe == 4
    q = sc.qe_array
    assert [q[k].type for k in range(4)] == [ffi.MIRROR, ffi.GRATING, ffi.MIRROR, ffi.DETECTOR]
    assert q[0].qe.n == 1 and q[0].qe.y[0] == 0.92
    g = q[1]
    assert (g.order, g.gr_const, g.alpha_deg, g.gamma_deg, g.blaze_deg) == (1, 1.0 / 0.6, 10.0, 0.0, 9.5)
    assert (g.rule_start, g.rule_stop) == (0.0, 0.2)
    x, y = S.qe_table()
    t = q[3].qe
    assert t.n == len(x)
    assert bits_equal([t.x[i] for i in range(t.n)], x) and bits_equal([t.y[i] for i in range(t.n)], y)
    assert bits_equal([t.y2[i] for i in range(t.n)], O.spline_init(x, y))


def test_committed_schemes_have_qe_surfaces():
    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rt_b200", "data")
    for fn, n in (("c0_littrow_free.xml", 4), ("c1_echelle.xml", 7), ("c4_littrow_free_flattener.xml", 5)):
        sc = S.LoadedScheme(os.path.join(here, fn))
        assert sc.qe_status == ffi.OK and sc.n_qe == n, fn


@pytest.mark.parametrize("edit,err", [
    (lambda s: setattr(s[0], "qe", None), 1),                          # no qe_curve: ParseFailure
    (lambda s: setattr(s[0], "qe", 0.0), 3),                           # TabulatedFunction::Set(<= 0)
    (lambda s: setattr(s[1], "rule_params", (0.7, 0.2)), 3),           # Grating::BadRuleParams
    (lambda s: setattr(s[1], "rule_params", (1.2, 1.5)), 3),           # clamped to 1, 1
])
def test_scheme_qe_errors(tmp_path, edit, err):
    specs = S.littrow_free()
    edit(specs)
    sc = S.LoadedScheme(write_scheme(tmp_path, specs))
    assert sc.status == ffi.OK          # the scheme still loads for ray tracing
    assert sc.qe_status == ffi.BAD_VALUE and sc.qe_error == err


def test_scheme_qe_missing_grating_attribute(tmp_path):
    path = write_scheme(tmp_path, S.littrow_free())
    text = open(path).read()
    open(path, "w").write(text.replace("<blaze_angle>9.5</blaze_angle>", ""))
    sc = S.LoadedScheme(path)
    assert sc.status == ffi.OK and sc.qe_error == 1


def test_scheme_without_qe_surfaces(tmp_path):
    """Only STOP and SHADE surfaces: ComputeQE's NoSurfaceDesc."""
    specs = [S.SurfaceSpec(ffi.PLANE, ffi.STOP, size=(10.0, 0.0)), S.SurfaceSpec(ffi.PLANE, ffi.SHADE, size=(1.0, 0.0))]
    sc = S.LoadedScheme(write_scheme(tmp_path, specs))
    assert sc.status == ffi.OK and sc.qe_error == 8


def test_qe_file_writer(tmp_path):
    L = ffi.load()
    L.rtb_save_qe.argtypes = [C.c_char_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(7)
    lam = rng.uniform(0.3, 0.9, size=(3, 17))
    qe = rng.uniform(0, 1, size=(3, 17))
    path = str(tmp_path / "qe.bin")
    assert L.rtb_save_qe(path.encode(), 3, 17, ffi.vptr(lam), ffi.vptr(qe)) == ffi.OK
    blocks = H.read_qe(path)
    assert len(blocks) == 3 and os.path.getsize(path) == 3 * (8 + 2 * 17 * 8)
    for r, (bl, bq) in enumerate(blocks):
        assert bits_equal(bl, lam[r]) and bits_equal(bq, qe[r])
    assert L.rtb_save_qe(str(tmp_path / "no" / "dir.bin").encode(), 3, 17, ffi.vptr(lam), ffi.vptr(qe)) != ffi.OK
