"""Throughput curves on the GPU (GPU tests): rtb_qe_curves, the one-launch
form of Scheme::ComputeQE's loop (common-lib/scheme.cpp:1249-1316), against
the per-surface drop-ins it fuses (same bits), the reference's own
cuda_engine on the same GPU (the same sin, cos and asin; the reference is
built with FMA contraction: within 1e-14 of each curve's largest value,
measured 7e-16), the oracle (host libm: qe_cases.tolerance), and the
rt_qe_comp program feeding rt_ccd_frame.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import pyoracle as O
import qe_cases as Q
import refharness as H
from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S
from test_qe import assert_curves_close, bits_equal

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "rt_b200", "bin")
CASES = Q.cases()
RT_PI = 3.14159265359


def drop_in_curves(cq, rows, n_lambda):
    """ComputeQE's loop over the drop-in calls rtb_surface_QE and
    rtb_grating_energy_distr, one call per surface and range, as the
    reference's Surface/Grating::ApplyQE make them."""
    L = E.lib()
    rows = np.atleast_2d(np.asarray(rows, dtype=np.float64))
    lam_all, qe_all = [], []
    for val in rows:
        d = (val[1] - val[0]) / (n_lambda - 1)
        lam = np.array([val[0] + d * i for i in range(n_lambda)])
        qe = np.ones(n_lambda)
        ig = 0
        for k in range(len(cq)):
            s = cq.array[k]
            ffi.check(L.rtb_surface_QE(n_lambda, ffi.vptr(lam), ffi.vptr(qe), C.byref(s.qe)), "rtb_surface_QE")
            if s.type != ffi.GRATING:
                continue
            order = int(val[2 + ig]) if rows.shape[0] > 1 else int(s.order)
            ig += 1
            a, b = (min(max(v, 0.0), 1.0) for v in (s.rule_start, s.rule_stop))
            ffi.check(L.rtb_grating_energy_distr(n_lambda, ffi.vptr(lam), abs(order), s.blaze_deg * RT_PI / 180.0,
                                                 s.alpha_deg * RT_PI / 180.0, s.gamma_deg * RT_PI / 180.0,
                                                 s.gr_const, a, b, ffi.vptr(qe)), "rtb_grating_energy_distr")
        lam_all.append(lam)
        qe_all.append(qe)
    return np.stack(lam_all), np.stack(qe_all)


@pytest.mark.parametrize("case", sorted(CASES))
def test_qe_curves_equal_the_drop_in_calls(case):
    specs, rows, n_lambda = CASES[case]
    cq = S.qe_surfaces(specs, E.spline_init)
    lam, qe = E.qe_curves(cq, rows, n_lambda)
    dl, dq = drop_in_curves(cq, rows, n_lambda)
    assert bits_equal(lam, dl)
    assert bits_equal(qe, dq) or (np.array_equal(np.isnan(qe), np.isnan(dq)) and
                                  bits_equal(qe[~np.isnan(qe)], dq[~np.isnan(dq)]))


@pytest.mark.parametrize("case", sorted(CASES))
def test_qe_curves_match_the_oracle(case):
    specs, rows, n_lambda = CASES[case]
    lam, qe = E.qe_curves(S.qe_surfaces(specs, E.spline_init), rows, n_lambda)
    ol, oq = O.qe_curves(S.qe_surfaces(specs, O.spline_init), rows, n_lambda)
    assert bits_equal(lam, ol)
    assert_curves_close(qe, oq, Q.tolerance(case))


@pytest.mark.skipif(H.harness("refgpu") is None, reason="reference cuda_engine harness not built")
@pytest.mark.parametrize("case", sorted(CASES))
def test_qe_curves_match_the_reference_cuda_engine(case):
    """The reference's host classes over its own cuda_engine on this GPU,
    and over this library's drop-ins (harness_b200, through the shim)."""
    specs, rows, n_lambda = CASES[case]
    specs = Q.scalar_qe(specs)
    rc, ref = H.run_qe("refgpu", specs, rows, n_lambda)
    assert rc == 0
    lam, qe = E.qe_curves(S.qe_surfaces(specs, E.spline_init), rows, n_lambda)
    assert bits_equal(lam, np.stack([b[0] for b in ref]))
    rq = np.stack([b[1] for b in ref])
    nan = np.isnan(rq)
    print(case, "identical:", np.mean(qe[~nan].view(np.uint64) == rq[~nan].view(np.uint64)),
          "max |B200 - reference| / max:", np.abs(qe[~nan] - rq[~nan]).max() / np.abs(rq[~nan]).max())
    assert_curves_close(qe, rq, 1e-14)
    if H.harness("b200") is not None:
        rc, shim = H.run_qe("b200", specs, rows, n_lambda)
        assert rc == 0
        sq = np.stack([b[1] for b in shim])
        assert np.array_equal(np.isnan(sq), np.isnan(qe))
        assert bits_equal(sq[~np.isnan(sq)], qe[~np.isnan(qe)])


def test_qe_curves_errors():
    x, y = S.qe_table()
    cq = S.qe_surfaces([S.SurfaceSpec(ffi.PLANE, ffi.MIRROR, qe=(x, y))], E.spline_init)
    with pytest.raises(RuntimeError, match="OUT_OF_RANGE"):
        E.qe_curves(cq, [[0.4, 0.8]], 33)
    cq = S.qe_surfaces([Q.grating(1, 1.0 / 0.6, 10.0, 0.0, 9.5, rule=(0.6, 0.3))], E.spline_init)
    with pytest.raises(RuntimeError, match="BAD_VALUE"):
        E.qe_curves(cq, [[0.4, 0.7]], 33)
    cq = S.qe_surfaces([S.SurfaceSpec(ffi.PLANE, ffi.MIRROR, qe=0.9)], E.spline_init)
    with pytest.raises(RuntimeError, match="BAD_VALUE"):
        E.qe_curves(cq, [[0.4, 0.7]], 1)        # one wavelength: the step divides by zero
    # more ranges than the grating orders in the rows
    cq = S.qe_surfaces(Q.qe_specs(S.echelle()), E.spline_init)
    with pytest.raises(RuntimeError, match="BAD_VALUE"):
        E.qe_curves(cq, [[0.4, 0.7], [0.5, 0.6]], 9)


def run(cmd, cwd):
    out = subprocess.run(cmd, cwd=str(cwd), capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return out


def test_rt_qe_comp_program(tmp_path):
    """rt_qe_comp on the committed echelle scheme (31 ranges from its range
    file, orders from the rows): the QE file holds rtb_qe_curves' curves."""
    xml = os.path.join(ROOT, "rt_b200", "data", "c1_echelle.xml")
    run([os.path.join(BIN, "rt_qe_comp"), xml, "129", "qe.bin"], tmp_path)
    blocks = H.read_qe(str(tmp_path / "qe.bin"))
    specs, rows, n = CASES["c1_ranges"]
    assert n == 129 and len(blocks) == len(rows)
    lam, qe = E.qe_curves(S.qe_surfaces(specs, E.spline_init), rows, n)
    assert bits_equal(np.stack([b[0] for b in blocks]), lam)
    assert bits_equal(np.stack([b[1] for b in blocks]), qe)
    ol, oq = O.qe_curves(S.qe_surfaces(specs, O.spline_init), rows, n)
    assert_curves_close(qe, oq, Q.tolerance("c1_ranges"))
    out = subprocess.run([os.path.join(BIN, "rt_qe_comp"), xml, "1", "qe.bin"], cwd=str(tmp_path),
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 1


def test_trace_qe_comp_ccd_frame_chain(tmp_path):
    """The reference's three programs in a row on C0: rt_trace writes the
    .dat file, rt_qe_comp the QE file, rt_ccd_frame the FITS image -- equal
    to the oracle's image from the same rays and the oracle's QE curve
    (1e-11: the curve's blaze factor, then sums in another order)."""
    xml = os.path.join(ROOT, "rt_b200", "data", "c0_littrow_free.xml")
    run([os.path.join(BIN, "rt_trace"), xml, "rt_files.txt", "log.txt", "--seed", "99"], tmp_path)
    files = [ln.strip() for ln in open(tmp_path / "rt_files.txt") if ln.strip()]
    (tmp_path / "rt_list.txt").write_text("".join(f + "\n" for f in files))
    run([os.path.join(BIN, "rt_qe_comp"), xml, "301", "qe.bin"], tmp_path)
    sx = np.linspace(0.3, 0.9, 13)
    S.write_table(str(tmp_path / "spec.txt"), sx, 1.0 + 0.5 * sx)
    c = S.C0_CCD
    (tmp_path / "ccd.txt").write_text(f"# CCD\n{c['xsize']} {c['ysize']}\n{c['xdim']} {c['ydim']}\n"
                                      f"{c['xpix']} {c['ypix']}\n")
    run([os.path.join(BIN, "rt_ccd_frame"), "rt_list.txt", "qe.bin", "spec.txt", "ccd.txt", "frame.fits"], tmp_path)
    raw = open(tmp_path / "frame.fits", "rb").read()
    img = np.frombuffer(raw[2880:2880 + 8 * c["xdim"] * c["ydim"]], dtype=">f8").reshape(c["ydim"], c["xdim"])
    # the oracle: its own QE curve and CCD image from the rays in the .dat file
    from test_gpu_runner import read_dat
    r, ng, _ = read_dat(str(tmp_path / files[0]))
    specs, rows, n = CASES["c0"]
    ol, oq = O.qe_curves(S.qe_surfaces(specs, O.spline_init), rows, n)
    Lo = O.load()
    cx, cy = np.zeros(ng, dtype=np.uint32), np.zeros(ng, dtype=np.uint32)
    Lo.oracle_ccd_coordinates(C.c_size_t(ng), ffi.dptr(r.X), ffi.dptr(r.Y), C.c_double(c["xsize"]),
                              C.c_double(c["ysize"]), C.c_double(c["xpix"]), C.c_double(c["ypix"]),
                              ffi.vptr(cx), ffi.vptr(cy))
    qt = ffi.TableHolder(x=ol[0], y=oq[0])
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
    np.testing.assert_allclose(img, ref, rtol=1e-11, atol=1e-11 * ref.max())
