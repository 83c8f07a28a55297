"""Edge cases of the fused plans (GPU tests): the largest scheme the engine
takes (RTB_MAX_SURFACES surfaces), one surface too many, and beams of zero,
one and a ragged number of rays in one plan -- each FP64 plan bit-identical to
the CPU oracle, each mixed plan's specialised kernel equal to the generic
kernel within the mixed engine's rounding."""
import ctypes as C

import numpy as np
import pytest
import torch

import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu

FIXES = ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP
TRACED = (ffi.OK, ffi.NO_INTERSECTIONS, ffi.NO_GOOD_RAYS)


def padded_lenses(n_total):
    """The lenses coverage scheme with pairs of AUX surfaces (a rotation
    about z and its inverse) between its surfaces, n_total surfaces in all."""
    base = S.coverage_schemes()["lenses"]
    n_aux = n_total - len(base)
    out = []
    for k, s in enumerate(base):
        out.append(s)
        while n_aux > 0 and len(out) < n_total - (len(base) - 1 - k):
            ang = 7.0 + len(out)
            out.append(S.SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE, angles=(0.0, 0.0, ang)))
            out.append(S.SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE, angles=(0.0, 0.0, -ang)))
            n_aux -= 2
    assert len(out) == n_total
    return out


def same_bits(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))


def fp64_plan_vs_oracle(specs, beams):
    n = S.total_rays(beams)
    cs_d, cs_o = S.to_c(specs, E.spline_init), S.to_c(specs, O.spline_init)
    plan = E.Plan(cs_d.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, fixes=FIXES))
    assert plan.specialized()[0]
    plan.run()
    st, stats = plan.result()
    ora = O.generate(beams, n)
    st_o, stats_o, _ = O.trace(cs_o.surfaces, beams, ora, fixes=FIXES)
    assert st == st_o and st in TRACED
    assert (stats.ray_surfaces, stats.n_good) == (stats_o.ray_surfaces, stats_o.n_good)
    out = E.device_view(plan.rays()[1])
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        assert same_bits(out[f].cpu().numpy(), getattr(ora, f)), f
    assert np.array_equal(out["flag"].cpu().numpy(), ora.flag)
    assert np.array_equal(out["lost_stage"].cpu().numpy(), ora.lost_stage)
    counts = plan.counts()
    plan.destroy()
    return stats, counts


def test_largest_scheme_fp64_plan_matches_oracle():
    specs = padded_lenses(RTB_MAX := 32)
    beams = [S.make_beam(0, 2000, 5, 10.0, (0.4, 0.8), 21)]
    stats, counts = fp64_plan_vs_oracle(specs, beams)
    assert stats.n_good > 0
    assert counts.shape == (1, 3 * RTB_MAX + 1) and int(counts.sum()) == beams[0].n_rays


def test_largest_scheme_mixed_specialised_equals_generic(monkeypatch):
    specs = padded_lenses(32)
    beams = [S.make_beam(0, 2000, 5, 10.0, (0.4, 0.8), 22)]
    cs = S.to_c(specs, E.spline_init)
    outs = []
    for spec in ("1", "0"):
        monkeypatch.setenv("RTB_SPECIALIZE", spec)
        plan = E.Plan(cs.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.MIXED, fixes=FIXES,
                                                  state_out=1))
        assert plan.specialized()[0] == (spec == "1")
        plan.run()
        st, stats = plan.result()
        outs.append((st, stats.n_good, {k: v.clone() for k, v in E.device_view(plan.rays()[1]).items()}))
        plan.destroy()
    (sa, ga, a), (sb, gb, b) = outs
    assert sa == sb and ga == gb > 0
    assert torch.equal(a["flag"], b["flag"]) and torch.equal(a["lost_stage"], b["lost_stage"])
    good = a["flag"] == 1
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        assert float((a[f][good] - b[f][good]).abs().max()) <= 1e-9, f


def test_one_surface_too_many_is_rejected():
    specs = padded_lenses(32) + [S.SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE)]
    cs = S.to_c(specs, E.spline_init)
    surf = (ffi.Surface * len(cs.surfaces))(*cs.surfaces)
    beams = [S.make_beam(0, 10, 1, 10.0, (0.5, 0.5), 1)]
    h = C.c_void_p()
    o = E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64)
    assert E.lib().rtb_plan_create(surf, len(surf), E._beams(beams), len(beams), C.byref(o), C.byref(h)) == \
        ffi.BAD_VALUE
    assert E.specialize(list(cs.surfaces), 0, ffi.MIXED)[0] == ffi.BAD_VALUE


def test_plan_with_empty_single_and_ragged_beams():
    """Beams of 0, 1, 37 and 1001 rays (orders of C1's echelle) in one plan:
    the empty beam counts nothing, every other ray is counted once, and the
    rays equal the oracle's bit for bit."""
    sizes = [(0, 1), (1, 1), (37, 1), (1001, 1)]
    beams, first = [], 0
    for k, (npl, nl) in enumerate(sizes):
        b = S.make_beam(first, max(npl, 1), nl, S.C1_RADIUS, (0.45 + 0.05 * k, 0.45 + 0.05 * k), 40 + k,
                        orders=(38 + k, 1))
        b.n_rays = npl
        b.disk[0] = float(max(npl, 1))
        beams.append(b)
        first += npl
    stats, counts = fp64_plan_vs_oracle(S.echelle(), beams)
    assert [int(r.sum()) for r in counts] == [npl for npl, _ in sizes]
