"""Batched plans (rtb_plan_*): many beams of uneven size, wavelength, field
angle and order in one graph-launched trace, and the autotuner (GPU tests).

* A plan's FP64 output equals the CPU oracle's trace of the same beams bit
  for bit; its mixed output equals rtb_trace_out's on the plan's own rays.
* Every launch configuration the autotuner tries gives the same result.
* The autotuner leaves the plan's frame untouched and its choice is reused
  by a later plan of the same scheme and size.
* The coherent tracing order (the default) and index order give the same
  rays, counters and frame.
* A mixed plan's kernel compiled for its scheme's structure gives the
  generic kernel's result bit for bit.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import ffi, metrics, schemes as S

pytestmark = pytest.mark.gpu

FIXES = ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP
TRACED = (ffi.OK, ffi.NO_INTERSECTIONS, ffi.NO_GOOD_RAYS)


def small_c3(n_beams=96, scale=0.004):
    """C3's beam draws with the ray counts scaled down (4..4000 per beam)."""
    return S.c3_beams(n_beams=n_beams, scale=scale)


def frame_opts(precision, ccd, block=0, rpt=0, state_out=0):
    counts = torch.zeros(int(ccd.xdim) * int(ccd.ydim), dtype=torch.int32, device="cuda")
    outside = torch.zeros(1, dtype=torch.int64, device="cuda")
    o = E.opts(engine=ffi.ENGINE_FUSED, precision=precision, fixes=FIXES, state_out=state_out, block=block, rpt=rpt,
               ccd=ccd, counts=counts, n_outside=outside)
    return o, counts, outside


def plan_output(plan):
    rin, rout = plan.rays()
    return E.device_view(rin), E.device_view(rout)


def test_plan_fp64_matches_oracle():
    beams = small_c3()
    n = S.total_rays(beams)
    cs_d, cs_o = S.to_c(S.echelle(), E.spline_init), S.to_c(S.echelle(), O.spline_init)
    plan = E.Plan(cs_d.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, fixes=FIXES))
    plan.run()
    st, stats = plan.result()
    ora = O.generate(beams, n)
    st_o, stats_o, _ = O.trace(cs_o.surfaces, beams, ora, fixes=FIXES)
    assert st == st_o
    assert (stats.ray_surfaces, stats.n_good) == (stats_o.ray_surfaces, stats_o.n_good)
    _, out = plan_output(plan)
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        a = out[f].cpu().numpy()
        b = getattr(ora, f)
        same = (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))
        assert same.all(), f
    assert np.array_equal(out["flag"].cpu().numpy(), ora.flag)
    assert np.array_equal(out["lost_stage"].cpu().numpy(), ora.lost_stage)
    plan.destroy()


@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32, ffi.FP64])
def test_plan_equals_trace_out_and_frame(precision):
    beams = small_c3()
    ccd = S.ccd(S.C1_CCD)
    cs = S.to_c(S.echelle(), E.spline_init)
    o, counts, outside = frame_opts(precision, ccd)
    plan = E.Plan(cs.surfaces, beams, o)
    plan.run()
    st, stats = plan.result()
    assert st in TRACED  # beams whose every ray is lost are reported, the rest traced
    rin, rout = plan_output(plan)
    # the same rays through rtb_trace_out
    n = S.total_rays(beams)
    src = E.DeviceRays(n)
    for f in E.FIELDS:
        getattr(src, f).copy_(rin[f])
    src.flag.copy_(rin["flag"])
    ref = E.DeviceRays(n)
    o2, counts2, outside2 = frame_opts(precision, ccd)
    stats2 = ffi.TraceStats()
    surf = (ffi.Surface * len(cs.surfaces))(*cs.surfaces)
    L = E.lib()
    L.rtb_trace_out.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                                C.POINTER(ffi.TraceOpts), C.POINTER(ffi.Rays), C.POINTER(ffi.Rays),
                                C.POINTER(ffi.TraceStats), C.c_void_p]
    st2 = L.rtb_trace_out(surf, len(surf), E._beams(beams), len(beams), C.byref(o2), C.byref(src.struct()),
                          C.byref(ref.struct()), C.byref(stats2), None)
    torch.cuda.synchronize()
    assert st2 == st
    assert (stats.ray_surfaces, stats.n_good) == (stats2.ray_surfaces, stats2.n_good)
    assert torch.equal(rout["X"], ref.X) and torch.equal(rout["Y"], ref.Y)
    assert torch.equal(rout["flag"], ref.flag) and torch.equal(rout["lost_stage"], ref.lost_stage)
    assert torch.equal(counts, counts2) and int(outside) == int(outside2)
    assert int(counts.sum()) + int(outside) == stats.n_good
    # per-beam counters: every ray of every beam accounted for once
    cnt = plan.counts()
    assert [int(r.sum()) for r in cnt] == [b.n_rays for b in beams]
    assert int(cnt[:, -1].sum()) == stats.n_good
    # a second run adds to the frame
    plan.run()
    assert plan.result()[0] == st
    assert torch.equal(counts, 2 * counts2)
    plan.destroy()


def test_plan_autotune_sweep_and_reuse():
    beams = small_c3(n_beams=64)
    ccd = S.ccd(S.C1_CCD)
    cs = S.to_c(S.echelle(), E.spline_init)
    o, counts, outside = frame_opts(ffi.MIXED, ccd)
    plan = E.Plan(cs.surfaces, beams, o)
    plan.run()
    st0, stats0 = plan.result()
    x0 = plan_output(plan)[1]["X"].clone()
    counts0 = counts.clone()
    table = plan.autotune(reps=2)
    assert len(table) == 12
    assert {(b, r) for b, r, _ in table} == {(b, r) for b in (128, 256, 512) for r in (1, 2, 4, 8)}
    assert all(ms > 0 for _, _, ms in table)
    assert torch.equal(counts, counts0)  # the sweep used its own frame
    best = min(table, key=lambda t: t[2])
    block, rpt, n = plan.config()
    assert (block, rpt) == best[:2] and n == S.total_rays(beams)
    plan.run()
    st1, stats1 = plan.result()
    assert st0 in TRACED and st1 == st0 and stats1.ray_surfaces == stats0.ray_surfaces
    assert torch.equal(plan_output(plan)[1]["X"], x0)
    # a second plan of the same scheme, precision, frame use and size starts tuned
    o2, _, _ = frame_opts(ffi.MIXED, ccd)
    plan2 = E.Plan(cs.surfaces, beams, o2)
    assert plan2.config()[:2] == (block, rpt)
    plan2.destroy()
    plan.destroy()


@pytest.mark.parametrize("block,rpt", [(128, 1), (512, 8), (256, 64)])
def test_plan_configs_agree(block, rpt):
    beams = small_c3(n_beams=48)
    cs = S.to_c(S.echelle(), E.spline_init)
    plan = E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=FIXES,
                                              state_out=1))
    plan.run()
    st0, ref_stats = plan.result()
    ref = {k: v.clone() for k, v in plan_output(plan)[1].items()}
    assert plan.set_config(block, rpt) == ffi.OK
    plan.run()
    st, stats = plan.result()
    assert st == st0 and st in TRACED and stats.ray_surfaces == ref_stats.ray_surfaces
    out = plan_output(plan)[1]
    for k in ("X", "Y", "Z", "cX", "cY", "cZ", "flag", "lost_stage"):
        assert torch.equal(out[k], ref[k]), k
    plan.destroy()


def test_plan_rejects_bad_requests():
    beams = small_c3(n_beams=8)
    cs = S.to_c(S.echelle(), E.spline_init)
    surf = (ffi.Surface * len(cs.surfaces))(*cs.surfaces)
    h = C.c_void_p()
    o = E.opts(engine=ffi.ENGINE_PER_SURFACE, precision=ffi.FP64)
    assert E.lib().rtb_plan_create(surf, len(surf), E._beams(beams), len(beams), C.byref(o), C.byref(h)) == \
        ffi.BAD_VALUE
    plan = E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64))
    assert plan.set_config(512, 2) == ffi.BAD_VALUE  # 512-thread blocks are for the mixed kernel
    assert plan.set_config(256, 0) == ffi.BAD_VALUE
    assert E.lib().rtb_plan_result(plan.h, None) == ffi.BAD_VALUE  # nothing ran yet
    plan.destroy()


@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32])
def test_plan_mixed_accuracy_on_c3(precision):
    """C3's mixed-precision run against the FP64 plan on the same beams."""
    beams = small_c3(n_beams=512, scale=0.02)
    cs = S.to_c(S.echelle(), E.spline_init)
    mk = lambda p: E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=p, fixes=FIXES))  # noqa
    pm, pr = mk(precision), mk(ffi.FP64)
    pm.run()
    pr.run()
    assert pm.result()[0] == pr.result()[0]
    assert pm.result()[0] in TRACED
    a, b = plan_output(pm)[1], plan_output(pr)[1]
    c = S.C1_CCD
    m = metrics.ccd_error(a["X"], a["Y"], a["flag"], b["X"], b["Y"], b["flag"], c["xsize"], c["ysize"], c["xpix"],
                          c["ypix"])
    print(m)
    assert m["rays_compared"] > 1000
    assert m["p99_9_um"] <= 0.05
    assert m["pixel_mismatch_rate"] < 1e-3
    pm.destroy()
    pr.destroy()


@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32, ffi.FP64])
@pytest.mark.parametrize("workload", ["c1", "c3"])
def test_plan_ray_order_does_not_change_results(precision, workload):
    """Plans trace their rays sorted by beam, wavelength and entrance
    position (RTB_ORDER_COHERENT) unless asked for index order; every output
    is the same either way."""
    beams = S.c1_beams(n_per_lambda=300) if workload == "c1" else small_c3()
    ccd = S.ccd(S.C1_CCD)
    cs = S.to_c(S.echelle(), E.spline_init)
    res = []
    for order in (ffi.ORDER_COHERENT, ffi.ORDER_INDEX):
        o, counts, outside = frame_opts(precision, ccd, state_out=1)
        o.ray_order = order
        plan = E.Plan(cs.surfaces, beams, o)
        plan.run()
        st, stats = plan.result()
        _, out = plan_output(plan)
        res.append((st, stats.ray_surfaces, stats.n_good, {k: v.clone() for k, v in out.items()}, counts.clone(),
                    int(outside), plan.counts()))
        plan.destroy()
    a, b = res
    assert a[:3] == b[:3] and a[0] in TRACED
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        x, y = a[3][f].view(torch.int64), b[3][f].view(torch.int64)
        assert torch.equal(x, y), f
    assert torch.equal(a[3]["flag"], b[3]["flag"]) and torch.equal(a[3]["lost_stage"], b[3]["lost_stage"])
    assert torch.equal(a[4], b[4]) and a[5] == b[5]
    assert np.array_equal(a[6], b[6])


def test_plan_rejects_unknown_ray_order():
    cs = S.to_c(S.echelle(), E.spline_init)
    o = E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=FIXES)
    o.ray_order = 7
    with pytest.raises(RuntimeError, match="BAD_VALUE"):
        E.Plan(cs.surfaces, small_c3(n_beams=4), o)


SPEC_SCHEMES = {
    "c0": (S.littrow_free, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c0_asphere": (S.c0_asphere_camera, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c4": (S.littrow_free_asphere, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c1": (S.echelle, dict(n_lambda=64, radius=25.0, lam_range=(0.38, 0.90)), (41, 1)),
    "mirrors": (lambda: S.coverage_schemes()["mirrors"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
    "lenses": (lambda: S.coverage_schemes()["lenses"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
    "gratings": (lambda: S.coverage_schemes()["gratings"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
}


@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32, ffi.FP64])
@pytest.mark.parametrize("name", sorted(SPEC_SCHEMES))
def test_specialised_plan_equals_generic_kernel(name, precision, monkeypatch):
    """A plan launches the kernel compiled for its scheme's structure; it
    computes what the generic kernel (RTB_SPECIALIZE=0) computes.  FP64: bit
    for bit (no contraction either way).  Mixed: the same lost flags, stages,
    counters and frame, and positions and cosines equal to 1e-9 (mm, or of a
    unit vector) -- bit for bit on most schemes, a few ulps apart where
    folding the scheme's branches lets the compiler contract a product and a
    sum into an FMA that the generic kernel keeps apart (the gratings
    scheme).  Both are far inside the mixed engine's 0.05 um budget against
    the FP64 oracle.  FP32 state: the contractions the compiler picks move
    the FP32 state by a few ulps, which the optics can amplify (a refraction
    near total internal reflection, on the lenses scheme, by up to 1e-3 mm on
    single rays): each kernel's CCD error against the FP64 engine (p99.9)
    stays within the FP32-state engine's bound for the scheme (0.05 um; the
    gratings scheme 0.15 um, the lenses scheme 1 um), and a ray on an aperture
    edge may fall on the other side (at most one in 1e4)."""
    make, kw, orders = SPEC_SCHEMES[name]
    beams = [S.make_beam(0, 3000, kw["n_lambda"], kw["radius"], kw["lam_range"], 11, orders=orders)]
    ccd = S.ccd(S.C1_CCD)
    cs = S.to_c(make(), E.spline_init)
    res = []
    for spec in ("1", "0"):
        monkeypatch.setenv("RTB_SPECIALIZE", spec)
        o, counts, outside = frame_opts(precision, ccd, state_out=1)
        plan = E.Plan(cs.surfaces, beams, o)
        on, note = plan.specialized()
        assert on == (spec == "1"), note
        plan.run()
        st, stats = plan.result()
        _, out = plan_output(plan)
        res.append((st, stats.ray_surfaces, stats.n_good, {k: v.clone() for k, v in out.items()}, counts.clone(),
                    int(outside), plan.counts()))
        plan.destroy()
    a, b = res
    assert a[0] == b[0] and a[0] in TRACED + (ffi.OUT_OF_RANGE,)
    assert a[2] > 0
    if precision == ffi.MIXED32:
        assert int((a[3]["flag"] != b[3]["flag"]).sum()) <= 1e-4 * a[3]["flag"].numel() + 1
        assert abs(a[2] - b[2]) <= 1e-4 * a[3]["flag"].numel() + 1
        o, counts64, outside64 = frame_opts(ffi.FP64, ccd, state_out=1)  # the plan writes into these
        plan = E.Plan(cs.surfaces, beams, o)
        torch.cuda.synchronize()  # the zeroed frame before the plan's own stream runs
        plan.run()
        plan.result()  # waits for the run
        _, ref = plan_output(plan)
        ref = {k: v.clone() for k, v in ref.items()}
        plan.destroy()
        torch.cuda.synchronize()
        del counts64, outside64

        def p999_um(out):
            both = (out["flag"] == 1) & (ref["flag"] == 1)
            d = torch.hypot(out["X"][both] - ref["X"][both], out["Y"][both] - ref["Y"][both]) * 1e3
            return float(torch.quantile(d.float().cpu(), 0.999))

        ea, eb = p999_um(a[3]), p999_um(b[3])
        print(name, "FP32 state, p99.9 um against FP64: specialised", ea, "generic", eb)
        bound = {"gratings": 0.15, "lenses": 1.0}.get(name, 0.05)
        assert max(ea, eb) <= bound, (ea, eb)
        return
    assert a[:3] == b[:3]
    same = 0
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        x, y = a[3][f], b[3][f]
        if precision == ffi.FP64:
            assert torch.equal(x.view(torch.int64), y.view(torch.int64)), f
        fin = torch.isfinite(x)
        assert torch.equal(fin, torch.isfinite(y)), f
        assert float((x[fin] - y[fin]).abs().max()) <= 1e-9, f
        same += int((x.view(torch.int64) == y.view(torch.int64)).sum())
    print(name, "bit-identical values:", same / (6 * x.numel()))
    assert torch.equal(a[3]["flag"], b[3]["flag"]) and torch.equal(a[3]["lost_stage"], b[3]["lost_stage"])
    assert torch.equal(a[4], b[4]) and a[5] == b[5]
    assert np.array_equal(a[6], b[6])


def test_plans_report_their_kernel(monkeypatch):
    cs = S.to_c(S.echelle(), E.spline_init)
    for prec in (ffi.FP64, ffi.MIXED, ffi.MIXED32):
        monkeypatch.setenv("RTB_SPECIALIZE", "1")
        plan = E.Plan(cs.surfaces, small_c3(n_beams=4), E.opts(engine=ffi.ENGINE_FUSED, precision=prec, fixes=FIXES))
        assert plan.specialized() == (True, "")
        plan.destroy()
        monkeypatch.setenv("RTB_SPECIALIZE", "0")
        plan = E.Plan(cs.surfaces, small_c3(n_beams=4), E.opts(engine=ffi.ENGINE_FUSED, precision=prec, fixes=FIXES))
        assert plan.specialized() == (False, "RTB_SPECIALIZE=0")
        plan.destroy()


def test_one_shot_trace_uses_a_compiled_specialisation(monkeypatch):
    """Once the kernel for a scheme's structure is compiled (rtb_specialize
    or a plan), rtb_trace_out launches it: on the gratings scheme, where the
    two kernels differ in the last bits, its output then equals the
    specialised plan's bit for bit."""
    monkeypatch.setenv("RTB_SPECIALIZE", "1")
    specs = S.coverage_schemes()["gratings"]
    beams = [S.make_beam(0, 3000, 5, 10.0, (0.4, 0.8), 11)]
    cs = S.to_c(specs, E.spline_init)
    st, note = E.specialize(list(cs.surfaces), FIXES)
    assert st == ffi.OK, note
    plan = E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=FIXES,
                                              state_out=1))
    assert plan.specialized()[0]
    plan.run()
    st_p, stats_p = plan.result()
    rin, rout = plan_output(plan)
    n = S.total_rays(beams)
    src = E.DeviceRays(n)
    for f in E.FIELDS:
        getattr(src, f).copy_(rin[f])
    src.flag.copy_(rin["flag"])
    ref = E.DeviceRays(n)
    o2 = E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=FIXES, state_out=1)
    stats2 = ffi.TraceStats()
    surf = (ffi.Surface * len(cs.surfaces))(*cs.surfaces)
    L = E.lib()
    L.rtb_trace_out.argtypes = [C.POINTER(ffi.Surface), C.c_size_t, C.POINTER(ffi.Beam), C.c_size_t,
                                C.POINTER(ffi.TraceOpts), C.POINTER(ffi.Rays), C.POINTER(ffi.Rays),
                                C.POINTER(ffi.TraceStats), C.c_void_p]
    st2 = L.rtb_trace_out(surf, len(surf), E._beams(beams), len(beams), C.byref(o2), C.byref(src.struct()),
                          C.byref(ref.struct()), C.byref(stats2), None)
    torch.cuda.synchronize()
    assert st2 == st_p and stats2.n_good == stats_p.n_good > 0
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        assert torch.equal(rout[f].view(torch.int64), getattr(ref, f).view(torch.int64)), f
    plan.destroy()


@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32, ffi.FP64])
def test_plan_outputs_by_slot(precision):
    """RTB_OUT_SLOT stores each ray's results at its tracing slot: the same
    values as RTB_OUT_INDEX, permuted by the plan's order (rtb_plan_order),
    with the same counters and frame."""
    beams = S.c1_beams(n_per_lambda=200)
    n = S.total_rays(beams)
    ccd = S.ccd(S.C1_CCD)
    cs = S.to_c(S.echelle(), E.spline_init)
    res = []
    for out_order in (ffi.OUT_INDEX, ffi.OUT_SLOT):
        o, counts, outside = frame_opts(precision, ccd, state_out=1)
        o.out_order = out_order
        plan = E.Plan(cs.surfaces, beams, o)
        plan.run()
        st, stats = plan.result()
        _, out = plan_output(plan)
        order = plan.order(n)
        res.append((st, stats.ray_surfaces, stats.n_good, {k: v.clone() for k, v in out.items()}, counts.clone(),
                    int(outside), order))
        plan.destroy()
    a, b = res
    assert a[:3] == b[:3] and a[0] in TRACED
    order = b[6]
    assert order is not None and torch.equal(order, a[6])
    assert torch.equal(torch.sort(order).values, torch.arange(n, device="cuda"))
    for f in ("X", "Y", "Z", "cX", "cY", "cZ", "flag", "lost_stage"):
        x, y = a[3][f][order], b[3][f]
        if x.dtype == torch.float64:
            x, y = x.view(torch.int64), y.view(torch.int64)
        assert torch.equal(x, y), f
    assert torch.equal(a[4], b[4]) and a[5] == b[5]


def frame_histogram(out, ccd):
    """The frame the mixed kernels accumulate, from a trace's own outputs: each
    good ray's pixel as the kernels compute it (coordinate plus half the CCD
    size, times the reciprocal pixel size, truncated with saturation)."""
    X, Y = out["X"].cpu().numpy(), out["Y"].cpu().numpy()
    good = out["flag"].cpu().numpy() == 1
    fin = good & np.isfinite(X) & np.isfinite(Y)

    def pix(v, size, p):
        t = (v + 0.5 * size) * (1.0 / p)
        return np.clip(np.nan_to_num(np.trunc(t), nan=0.0), 0, 2.0**32 - 1)

    ix, iy = pix(X[fin], ccd.xsize, ccd.xpix), pix(Y[fin], ccd.ysize, ccd.ypix)
    inside = (ix < ccd.xdim) & (iy < ccd.ydim)
    p = iy[inside].astype(np.int64) * int(ccd.xdim) + ix[inside].astype(np.int64)
    hist = np.bincount(p, minlength=int(ccd.xdim) * int(ccd.ydim)).astype(np.uint32)
    return hist, int(good.sum() - inside.sum())


@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32])
def test_mixed_plan_frame_is_the_histogram_of_its_outputs(precision):
    """A mixed plan's frame counts equal the histogram of the plan's own
    detector coordinates, run after run, for a frame at any 4-byte alignment
    and of any size, and it writes nothing outside the frame."""
    beams = S.c1_beams(n_per_lambda=200)
    cs = S.to_c(S.echelle(), E.spline_init)
    c1 = S.ccd(S.C1_CCD)
    odd = ffi.CCD(c1.xsize, c1.ysize, 4095, 4095, c1.xpix, c1.ypix)  # an odd number of pixels
    for ccd, offset in ((c1, 0), (c1, 1), (odd, 0)):
        n_pix = int(ccd.xdim) * int(ccd.ydim)
        buf = torch.zeros(n_pix + 4, dtype=torch.int32, device="cuda")
        counts = buf[offset:offset + n_pix]  # offset 1: 4-byte aligned only
        outside = torch.zeros(1, dtype=torch.int64, device="cuda")
        o = E.opts(engine=ffi.ENGINE_FUSED, precision=precision, fixes=FIXES, ccd=ccd, counts=counts,
                   n_outside=outside)
        plan = E.Plan(cs.surfaces, beams, o)
        torch.cuda.synchronize()  # the zeroed frame, before the plan's own stream adds to it
        plan.run()
        st, stats = plan.result()
        assert st in TRACED and stats.n_good > 0
        _, out = plan_output(plan)
        hist, n_out = frame_histogram(out, ccd)
        got = counts.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, hist), (ccd.xdim, offset, int((got != hist).sum()))
        assert int(outside) == n_out
        plan.run()
        assert plan.result()[0] == st
        assert np.array_equal(counts.cpu().numpy().view(np.uint32), 2 * hist)
        # nothing written outside the frame
        assert int(buf[:offset].abs().sum()) == 0 and int(buf[offset + n_pix:].abs().sum()) == 0
        plan.destroy()
