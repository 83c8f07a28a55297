"""The benchmark workloads at their full sizes, checked through properties that
do not depend on the size (GPU tests; a few GB of device memory, seconds).

* C1 (1.0e8 rays, 31 echelle orders x 64 wavelengths, frame counts), as the
  bench runs it, in the plain FP64 plan and the FP64-state mixed plan:
  every ray is counted exactly once (per beam, the loss counters and the
  good count add up to the beam's rays), the frame holds every good ray
  (pixel counts + rays outside the frame = good rays), a second run gives
  the same bits, the tracing order is a permutation of the rays, and the
  mixed plan stays within 0.05 um (p99.9) of the FP64 plan's CCD positions.
* C3 (512 beams, 7.4e7 rays, one launch): the same conservation laws.
* C4 (1e7 rays, 24 parameters): the reverse sweep's merit gradient equals
  the forward-mode passes' to 1e-12 relative.
"""
import numpy as np
import pytest
import torch

from rt_b200 import engine as E
from rt_b200 import ffi, metrics, schemes as S

pytestmark = pytest.mark.gpu

FIXES = ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP


def _run_plan(cs, beams, precision, ccd, out_order=ffi.OUT_INDEX):
    counts = torch.zeros(int(ccd.xdim) * int(ccd.ydim), dtype=torch.int32, device="cuda")
    outside = torch.zeros(1, dtype=torch.int64, device="cuda")
    o = E.opts(engine=ffi.ENGINE_FUSED, precision=precision, fixes=FIXES, state_out=0, ccd=ccd, counts=counts,
               n_outside=outside, out_order=out_order)
    plan = E.Plan(cs.surfaces, beams, o)
    return plan, counts, outside


def _conserved(plan, beams, counts, outside):
    st, stats = plan.result()
    assert st in (ffi.OK, ffi.NO_INTERSECTIONS, ffi.NO_GOOD_RAYS)
    c = plan.counts()
    per_beam = c.sum(axis=1)
    assert np.array_equal(per_beam, np.array([b.n_rays for b in beams], dtype=np.uint64))
    assert int(c[:, -1].sum()) == stats.n_good
    torch.cuda.synchronize()
    assert int(counts.sum()) + int(outside.item()) == stats.n_good
    return stats


def _outputs(plan):
    out = E.device_view(plan.rays()[1])
    return {k: out[k].clone() for k in ("X", "Y", "flag")}


def test_c1_full_size_conservation_determinism_and_accuracy():
    beams = S.c1_beams()  # 31 x 64 x 50404 = 1.0e8 rays
    n = S.total_rays(beams)
    assert n > 9.9e7
    cs = S.to_c(S.echelle(), E.spline_init)
    ccd = S.ccd(S.C1_CCD)
    outs = {}
    for prec in (ffi.FP64, ffi.MIXED):
        plan, counts, outside = _run_plan(cs, beams, prec, ccd)
        torch.cuda.synchronize()  # the zeroed frame, before the library's stream uses it
        plan.run()
        stats = _conserved(plan, beams, counts, outside)
        first = _outputs(plan)
        frame = counts.clone()
        counts.zero_()
        outside.zero_()
        torch.cuda.synchronize()  # the plan runs on the library's own stream
        plan.run()
        _conserved(plan, beams, counts, outside)
        again = _outputs(plan)
        for k in ("X", "Y"):
            assert torch.equal(first[k].view(torch.int64), again[k].view(torch.int64)), (prec, k)
        assert torch.equal(first["flag"], again["flag"]) and torch.equal(frame, counts), prec
        outs[prec] = (first, stats.n_good)
        plan.destroy()
        del counts, outside, frame, again
        torch.cuda.empty_cache()
    (f, gf), (m, gm) = outs[ffi.FP64], outs[ffi.MIXED]
    c = S.C1_CCD
    acc = metrics.ccd_error(m["X"], m["Y"], m["flag"], f["X"], f["Y"], f["flag"], c["xsize"], c["ysize"], c["xpix"],
                            c["ypix"])
    print("C1 full size, mixed against FP64:", acc)
    assert acc["rays_compared"] > 0.3 * n
    assert acc["p99_9_um"] <= 0.05
    assert acc["pixel_mismatch_rate"] < 1e-3
    assert abs(gf - gm) <= 1e-6 * n + 2
    del outs, f, m
    torch.cuda.empty_cache()


def test_c1_full_size_tracing_order_is_a_permutation():
    beams = S.c1_beams()
    n = S.total_rays(beams)
    cs = S.to_c(S.echelle(), E.spline_init)
    plan = E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=FIXES,
                                             state_out=0, out_order=ffi.OUT_SLOT))
    plan.run()
    order = plan.order(n)
    assert order is not None and order.numel() == n
    srt, _ = torch.sort(order)
    assert torch.equal(srt, torch.arange(n, device="cuda", dtype=torch.int64))
    # beam-major: each beam's rays occupy its own contiguous run of slots
    firsts = torch.tensor([b.first_ray for b in beams] + [n], device="cuda", dtype=torch.int64)
    beam_of_slot = torch.bucketize(order, firsts[1:], right=True)
    assert bool((beam_of_slot[1:] >= beam_of_slot[:-1]).all())
    plan.destroy()
    del order, srt, beam_of_slot
    torch.cuda.empty_cache()


def test_c3_full_size_conservation():
    beams = S.c3_beams()
    n = S.total_rays(beams)
    assert n > 5e7
    cs = S.to_c(S.echelle(), E.spline_init)
    ccd = S.ccd(S.C1_CCD)
    plan, counts, outside = _run_plan(cs, beams, ffi.MIXED, ccd, out_order=ffi.OUT_SLOT)
    torch.cuda.synchronize()
    plan.run()
    stats = _conserved(plan, beams, counts, outside)
    assert stats.n_good > 0
    plan.destroy()
    del counts, outside
    torch.cuda.empty_cache()


def test_c4_full_size_reverse_sweep_equals_passes(monkeypatch):
    beams = S.c4_beams()  # 64 x 156250 = 1e7 rays
    n = S.total_rays(beams)
    cs = S.to_c(S.littrow_free_asphere(), E.spline_init)
    rays = E.generate(beams, n)
    adj = E.Adjoint(cs.surfaces, S.c4_params(), beams, n, fixes=ffi.FIX_ASPHERE_ROOT)
    st, _ = adj.forward(None, rays)
    assert st == ffi.OK
    lam = np.linspace(S.C4_LAMBDA[0], S.C4_LAMBDA[1], S.C4_NLAMBDA)
    _, gX, gY = adj.spot_merit(S.c4_target_x(lam), 10.0)
    monkeypatch.delenv("RTB_ADJOINT_BACKWARD", raising=False)
    g_rev = adj.backward(gX, gY)
    monkeypatch.setenv("RTB_ADJOINT_BACKWARD", "passes")
    g_pas = adj.backward(gX, gY)
    rel = np.abs(g_rev - g_pas) / np.abs(g_pas)
    print("C4 full size: reverse vs passes, max rel", rel.max())
    assert rel.max() <= 1e-12
    adj.destroy()
    del rays, gX, gY
    torch.cuda.empty_cache()
