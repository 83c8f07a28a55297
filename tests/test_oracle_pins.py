"""Pins of the CPU oracle (no GPU needed).

* The oracle's literal replica of the per-surface loop equals, bit for bit,
  the reference's own host classes (Beam, Surface, TabulatedFunction compiled
  from the reference sources) driving the same engine math
  (oracle/_ref/harness_cpu).  This pins Normalize, Rearrange,
  ApplyConstrains, the transform plumbing, the angle round trip and the
  exception behaviour to the reference.
* The per-ray formulation (what the B200 engine computes) equals the literal
  replica once rays are put in the reference's order and lost rays are
  re-normalised.
"""
import numpy as np
import pytest

import pyoracle as O
import refharness as H
from rt_b200 import ffi, schemes as S

CASES = {
    "c0": (S.littrow_free, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c4": (S.littrow_free_asphere, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c1_m30": (S.echelle, dict(n_lambda=64, radius=25.0, lam_range=(0.38, 0.90)), (30, 1)),
    "c1_m47": (S.echelle, dict(n_lambda=64, radius=25.0, lam_range=(0.38, 0.90)), (47, 1)),
    "mirrors": (lambda: S.coverage_schemes()["mirrors"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
    "lenses": (lambda: S.coverage_schemes()["lenses"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
    "gratings": (lambda: S.coverage_schemes()["gratings"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
}


def _beam(case, n_per=60, seed=123):
    make, kw, orders = CASES[case]
    b = S.make_beam(0, n_per, kw["n_lambda"], kw["radius"], kw["lam_range"], seed, orders=orders)
    return make(), b


def same_bits(a, b):
    """Bit-identical, except that any NaN equals any NaN (IEEE 754 leaves the
    sign and payload of a NaN result unspecified)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    eq = a.view(np.uint64) == b.view(np.uint64)
    return bool(np.all(eq | (np.isnan(a) & np.isnan(b))))


@pytest.mark.parametrize("case", list(CASES))
def test_literal_equals_reference_host_classes(case):
    if H.harness("cpu") is None:
        pytest.skip("oracle/_ref/harness_cpu not built (reference sources absent)")
    specs, beam = _beam(case)
    rays = O.generate([beam], beam.n_rays)
    ref_rc, ref = H.run_trace("cpu", specs, list(beam.orders)[:beam.n_orders], rays)
    lit = rays.copy()
    cs = S.to_c(specs, O.spline_init)
    st, ng = O.trace_literal(cs.surfaces, beam, lit)
    assert ref_rc == st
    if st != ffi.OK:
        return
    n, ref_ng, _, ref_state = ref
    assert ref_ng == ng and n == beam.n_rays
    ours = np.stack([lit.X, lit.Y, lit.Z, lit.cX, lit.cY, lit.cZ, lit.lambda_])
    assert same_bits(ours, ref_state)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("fixes", [0, ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP, 7])
def test_per_ray_equals_literal(case, fixes):
    specs, beam = _beam(case, n_per=80, seed=7)
    cs = S.to_c(specs, O.spline_init)
    rays = O.generate([beam], beam.n_rays)
    lit = rays.copy()
    st_l, ng = O.trace_literal(cs.surfaces, beam, lit, fixes=fixes)
    st_p, stats, counts = O.trace(cs.surfaces, [beam], rays, fixes=fixes)
    assert st_l == st_p
    if st_p != ffi.OK:
        return
    order, ng2 = O.reference_order(rays.lost_stage, 3 * len(specs))
    assert ng2 == ng == stats.n_good
    perm = rays.take(order)
    for f in ("X", "Y", "Z", "cX", "cY", "cZ", "lambda_"):
        assert same_bits(getattr(perm, f), getattr(lit, f)), f
    assert np.array_equal(perm.flag, lit.flag)
    # ray-surfaces: lost rays count their losing surface
    nonaux_upto = np.cumsum([s.type != ffi.AUX_TYPE for s in specs])
    ls = rays.lost_stage.astype(int)
    expect = np.where(ls == ffi.NOT_LOST, nonaux_upto[-1], nonaux_upto[np.minimum(ls // 3, len(specs) - 1)]).sum()
    assert stats.ray_surfaces == expect


def test_lost_counts_match_flags():
    specs, beam = _beam("c1_m47", n_per=100)
    cs = S.to_c(specs, O.spline_init)
    rays = O.generate([beam], beam.n_rays)
    st, stats, counts = O.trace(cs.surfaces, [beam], rays)
    assert st == ffi.OK
    hist = np.bincount(rays.lost_stage[rays.lost_stage != ffi.NOT_LOST], minlength=3 * len(specs))
    assert np.array_equal(hist, counts[0])
    assert stats.n_good == int((rays.flag == 1).sum())


def test_no_intersections_status():
    """A scheme whose first surface lies behind the beam loses every ray at
    the first intersection: the reference throws NoIntersections."""
    specs = [S.SurfaceSpec(ffi.PLANE, ffi.DETECTOR, distance=(0.0, 0.0, -10.0))]
    beam = S.make_beam(0, 10, 1, 5.0, (0.5, 0.5), 1)
    cs = S.to_c(specs, O.spline_init)
    rays = O.generate([beam], beam.n_rays)
    st, stats, _ = O.trace(cs.surfaces, [beam], rays)
    assert st == ffi.NO_INTERSECTIONS and stats.failed_stage == 0
    if H.harness("cpu") is not None:
        rc, _ = H.run_trace("cpu", specs, [], rays)
        assert rc == ffi.NO_INTERSECTIONS


def _toric_with_cycle_skip(r, c, k1, cR, fix_sign, fix_step):
    """Scalar restatement of the CUDA engine's toric iteration: the
    reference's Steffensen loop (rt_cuda_engine_surface.cu:359-410) plus the
    engine's exact skip of whole periods once the state (sn1, Fyn) repeats
    bit for bit (Brent's cycle finding, armed after 8 steps)."""
    import math
    import struct
    X0, Y0, Z0, cX, cY, cZ = r
    sgn = -1.0 if fix_sign else 1.0

    def F(t):
        X, Y, Z = X0 + t * cX, Y0 + t * cY, Z0 + t * cZ
        Y2 = Y * Y
        FY = c * Y2 / (1.0 + math.sqrt(1.0 + sgn * k1 * c * c * Y2))
        return Z - FY - 0.5 * cR * (X * X + Z * Z - FY * FY)

    bits = lambda v: struct.pack("<d", v)  # noqa: E731
    sn1 = -Z0 / cZ
    if not sn1 >= 0:
        return None, 0
    niter, Fyn, skipped = 0, 0.0, 0
    saved, power, lam, armed = None, 1, 0, False
    while True:
        sn = sn1
        Fxn = F(sn)
        if abs(Fyn - Fxn) <= 1e-7:
            break
        Fzn = F(sn + Fxn)
        if fix_step and Fzn - Fxn == 0.0:
            sn1 = sn
            break
        sn1 = sn - Fxn * Fxn / (Fzn - Fxn)
        Fyn = Fxn
        niter += 1
        if niter >= 8:
            key = bits(sn1) + bits(Fyn)
            if not armed:
                armed, saved = True, key
            else:
                lam += 1
                if key == saved:
                    left = 100000 + 1 - niter
                    niter += left - left % lam
                    skipped += left - left % lam
                elif lam == power:
                    saved, power, lam = key, power * 2, 0
        if not (abs(sn1 - sn) >= 1e-7 and niter <= 100000):
            break
    return (X0 + sn1 * cX, Y0 + sn1 * cY, Z0 + sn1 * cZ), skipped


@pytest.mark.parametrize("fixes", [0, ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP])
def test_toric_cycle_skip_equals_full_iteration(fixes):
    """The rays of the C1 fold that cycle until the iteration cap
    (tests/golden/toric_cycles.npz): skipping whole periods gives the bits of
    the oracle's full 1e5-step loop."""
    import ctypes as C
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "toric_cycles.npz"))
    st = z["state"]
    n = st.shape[1]
    r = O.HostRays(n)
    for f, row in zip(O.HostRays.FIELDS[:6], st):
        getattr(r, f)[:] = row
    p = np.zeros(16)
    p[:4] = z["params"][:4]
    nb = C.c_size_t(0)
    assert O.load().oracle_surface_intersection_fix(
        ffi.TORIC, ffi.dptr(p), C.c_size_t(n), *(ffi.dptr(getattr(r, f)) for f in O.HostRays.FIELDS[:6]),
        C.byref(nb), ffi.vptr(r.flag), C.c_uint(fixes)) == ffi.OK
    c, k, _, cR = z["params"][:4]
    n_skipped = 0
    for i in range(n):
        xyz, skipped = _toric_with_cycle_skip(st[:, i], c, k + 1.0, cR, bool(fixes & ffi.FIX_TORIC_SIGN),
                                              bool(fixes & ffi.FIX_TORIC_STEP))
        n_skipped += skipped > 0
        assert xyz is not None and r.flag[i] == 1
        assert same_bits(np.array(xyz), np.array([r.X[i], r.Y[i], r.Z[i]])), i
    cyc = z["cycling_fixed"] if fixes else z["cycling_literal"]
    assert n_skipped == int(cyc.sum()) >= 1
