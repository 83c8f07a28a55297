"""Finds the C1 rays whose toric fold iteration never converges.

The reference's Steffensen iteration (cuda_engine/rt_cuda_engine_surface.cu:
359-410) stops on convergence or after ITER_MAX = 100000 steps.  On the C1
echelle's toric fold, 5 of the 8.7e7 rays that reach it fall into an exact
2-cycle and run to the cap; the CUDA engine skips such cycles in whole periods
and must still return the same bits.  This script traces C1's first three
surfaces with the CPU oracle, finds the rays whose iteration -- with the
reference's sign of the sag term, or with the fixed one -- is still running
after 60 steps, and stores their state in the toric's local frame, plus a few
converging neighbours, in tests/golden/toric_cycles.npz.  CPU only; takes a
few minutes.

  python tests/golden/make_toric_cycles.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

import pyoracle as O  # noqa: E402
from rt_b200 import ffi, schemes as S  # noqa: E402

EPS = 1e-7


def steffensen_active(st, c, k1, cR, fix_sign, steps=60):
    """Vectorised restatement of the toric iteration; True where a ray is
    still iterating after `steps`."""
    X0, Y0, Z0, cX, cY, cZ = st
    sgn = 1.0 if fix_sign else -1.0

    def F(t):
        X, Y, Z = X0 + t * cX, Y0 + t * cY, Z0 + t * cZ
        Y2 = Y * Y
        FY = c * Y2 / (1.0 + np.sqrt(1.0 - sgn * k1 * c * c * Y2))
        return Z - FY - 0.5 * cR * (X * X + Z * Z - FY * FY)

    with np.errstate(all="ignore"):
        sn1 = -Z0 / cZ
        Fyn = np.zeros_like(sn1)
        active = sn1 >= 0
        for _ in range(steps):
            sn = sn1.copy()
            Fxn = F(sn)
            active &= ~(np.abs(Fyn - Fxn) <= EPS)
            den = F(sn + Fxn) - Fxn
            active &= ~(den == 0)
            sn1 = np.where(active, sn - Fxn * Fxn / den, sn1)
            Fyn = np.where(active, Fxn, Fyn)
            active &= np.abs(sn1 - sn) >= EPS
    return active


def main(out=os.path.join(HERE, "toric_cycles.npz")):
    specs = S.echelle()
    toric = specs[3]
    assert toric.cls == ffi.TORIC
    aux = S.SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE, distance=toric.distance, angles=toric.angles)
    cs = S.to_c(specs[:3] + [aux], O.spline_init)
    c, k, _, cR = toric.params[:4]
    beams = S.c1_beams(n_per_lambda=S.c1_rays_per_lambda())
    rng = np.random.default_rng(7)
    picked, fixed, literal = [], [], []
    for bi, b in enumerate(beams):
        b.first_ray = 0
        rays = O.generate([b], S.total_rays([b]))
        O.trace(cs.surfaces, [b], rays)
        good = np.nonzero(rays.flag == 1)[0]
        st = rays.state()[:, good]
        a_fix = steffensen_active(st, c, k + 1.0, cR, True)
        a_lit = steffensen_active(st, c, k + 1.0, cR, False)
        act = np.nonzero(a_fix | a_lit)[0]
        print("beam", bi, "cycling rays", int(a_fix.sum()), int(a_lit.sum()), flush=True)
        if not len(act):
            continue
        near = rng.choice(len(good), 16, replace=False)
        idx = np.concatenate([act, near])
        picked.append(st[:, idx])
        fixed.append(a_fix[idx])
        literal.append(a_lit[idx])
    st = np.concatenate(picked, axis=1)
    np.savez_compressed(out, state=st, params=np.array(toric.params, dtype=np.float64),
                        cycling_fixed=np.concatenate(fixed), cycling_literal=np.concatenate(literal))
    print("wrote", out, st.shape)


if __name__ == "__main__":
    main()
