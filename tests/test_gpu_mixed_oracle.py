"""Both mixed-precision engines against the CPU oracle directly (GPU tests).

The mixed plans (RTB_MIXED: FP64 ray state; RTB_MIXED32: FP32 ray state)
trace a fixed sample of C1 -- every one of the 31 echelle orders, all 64
wavelengths -- and of C3's beam draws, and the oracle traces the same
generated rays on the CPU.  Checked: the CCD error of rays good in both
(p99.9 <= 0.05 um; for the FP64-state engine also p99.9 <= 0.01 um and max
<= 0.02 um, its own precision), the pixel mismatch rate, and which rays are
lost.

In the reference's own quirk mode (fixes = 0) the FP64 toric iteration
divides 0/0 once converged (iter_toric, rt_cuda_engine_surface.cu:390) and
sends about a quarter of the rays that reach C1's fold to NaN, which the lens
then loses.  The mixed engines solve the toric by Newton and do not meet that
division, so those rays survive in them.  The test reports that mismatch and
checks that it is all of this kind: every ray good in a mixed engine and lost
by the oracle has a NaN position in the oracle's trace and was lost after the
fold; no ray is good in the oracle and lost by a mixed engine beyond the
aperture-edge rate.
"""
import numpy as np
import pytest
import torch

import pyoracle as O
from rt_b200 import engine as E
from rt_b200 import ffi, metrics, schemes as S

pytestmark = pytest.mark.gpu

FOLD = 3  # index of C1's toric fold


def _workload(name):
    if name == "c1":
        return S.c1_beams(n_per_lambda=100)  # 31 x 64 x 100 = 198,400 rays
    return S.c3_beams(n_beams=512, scale=0.004)


@pytest.mark.parametrize("fixes", [3, 0])
@pytest.mark.parametrize("precision", [ffi.MIXED, ffi.MIXED32])
@pytest.mark.parametrize("workload", ["c1", "c3"])
def test_mixed_plan_against_oracle(workload, precision, fixes):
    beams = _workload(workload)
    n = S.total_rays(beams)
    cs_d, cs_o = S.to_c(S.echelle(), E.spline_init), S.to_c(S.echelle(), O.spline_init)
    plan = E.Plan(cs_d.surfaces, beams, E.opts(engine=ffi.ENGINE_FUSED, precision=precision, fixes=fixes,
                                                state_out=0))
    plan.run()
    st, stats = plan.result()
    assert st in (ffi.OK, ffi.NO_INTERSECTIONS, ffi.NO_GOOD_RAYS)
    out = E.device_view(plan.rays()[1])
    mx, my = out["X"].cpu().numpy(), out["Y"].cpu().numpy()
    mf, ms = out["flag"].cpu().numpy(), out["lost_stage"].cpu().numpy()
    plan.destroy()

    ora = O.generate(beams, n)
    O.trace(cs_o.surfaces, beams, ora, fixes=fixes)
    c = S.C1_CCD
    m = metrics.ccd_error(mx, my, mf, ora.X, ora.Y, ora.flag, c["xsize"], c["ysize"], c["xpix"], c["ypix"])
    good_m, good_o = mf == 1, ora.flag == 1
    only_m = good_m & ~good_o
    only_o = good_o & ~good_m
    print(workload, precision, fixes, m, "good only in mixed:", int(only_m.sum()), "only in oracle:",
          int(only_o.sum()))
    assert m["rays_compared"] > 0.05 * n
    assert m["p99_9_um"] <= 0.05
    if precision == ffi.MIXED:
        # the FP64-state engine's error comes from its FP32 normals (~0.005 um
        # at p99.9 on C1): a guard on its precision, well inside the budget
        assert m["p99_9_um"] <= 0.01 and m["max_um"] <= 0.02, m
    assert int(only_o.sum()) <= 2e-5 * n + 2  # aperture-edge rays
    if fixes & ffi.FIX_TORIC_STEP:
        assert m["pixel_mismatch_rate"] < 1e-3
        assert int(only_m.sum()) <= 2e-5 * n + 2
    else:
        # the reference's toric 0/0: lost by the oracle after the fold with a NaN position
        nan_o = np.isnan(ora.X) | np.isnan(ora.Y)
        assert np.all(nan_o[only_m]), "a ray lost by the oracle is not explained by the toric 0/0"
        assert np.all(ora.lost_stage[only_m] >= 3 * (FOLD + 1))
        print(f"{workload}: toric 0/0 mismatch rate {only_m.sum() / max(1, good_m.sum()):.4f}")
