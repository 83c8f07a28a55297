"""Generates the golden fixtures of the reference CUDA engine.

Runs oracle/_ref/harness_refgpu -- the reference's Beam/Surface/
TabulatedFunction host classes over the reference's own cuda_engine compiled
for sm_100a (oracle/Makefile) -- on small seeded beams through the benchmark
and coverage schemes, and stores input and output of each case in
tests/golden/<case>.npz.  The *_nofma cases run the same sources built
without FMA contraction (harness_refgpu_nofma).  Needs a GPU; the fixtures are committed so that the
CPU tests can pin the oracle to the reference engine without one.

Lens and grating refractive indices are single values in these cases: the
reference's spline_init kernel runs the natural-spline recurrence in parallel
(rt_cuda_engine_spline.cu:21-37) and returns racy second derivatives, so
tabulated indices would not be a reproducible fixture.

  python tests/golden/make_golden.py [out_dir] [--only=case1,case2]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import pyoracle as O  # noqa: E402
import refharness as H  # noqa: E402
from rt_b200 import ffi, schemes as S  # noqa: E402


def scalarize(specs, value=1.5):
    """Replace tabulated indices by single values (see module doc)."""
    out = []
    for s in specs:
        s = S.SurfaceSpec(**s.__dict__)
        if not isinstance(s.n1, (int, float)):
            s.n1 = value
        if not isinstance(s.n2, (int, float)):
            s.n2 = value
        out.append(s)
    return out


def sphere_fold(specs):
    """C1 with the toric fold replaced by a sphere of the mean radius: the
    reference's toric iteration divides 0/0 for rays that converge exactly
    (surface.cu:390), and which rays do depends on FMA contraction, so the
    toric-free variant pins everything else ray by ray."""
    out = []
    for s in specs:
        s = S.SurfaceSpec(**s.__dict__)
        if s.cls == ffi.TORIC:
            s.cls = ffi.CONIC
            s.params = (-1 / 2050.0, 0.0, 0)
        out.append(s)
    return out


def cases():
    cov = S.coverage_schemes()
    c0 = dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7))
    c1 = dict(n_lambda=64, radius=25.0, lam_range=(0.38, 0.90))
    small = dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8))
    c4 = dict(n_lambda=64, radius=10.0, lam_range=(0.4, 0.7))
    return {
        "c0": (S.littrow_free(), c0, (), 400),
        "c0_asphere_camera": (S.c0_asphere_camera(), c0, (), 400),
        "c4": (scalarize(S.littrow_free_asphere()), c4, (), 100),
        "c1_m38": (scalarize(S.echelle()), c1, (38, 1), 40),
        "c1_m52": (scalarize(S.echelle()), c1, (52, 1), 40),
        "c1_sphere_m38": (sphere_fold(scalarize(S.echelle())), c1, (38, 1), 40),
        "c1_sphere_m52": (sphere_fold(scalarize(S.echelle())), c1, (52, 1), 40),
        "mirrors": (cov["mirrors"], small, (), 400),
        "mirrors_tagged": (cov["mirrors"], small, (), 400),
        "lenses": (scalarize(cov["lenses"]), small, (), 400),
        "gratings": (scalarize(cov["gratings"]), small, (), 400),
        # C1 with its toric fold, through the reference built without FMA
        # contraction (HARNESS): the same rays meet the toric step's 0/0 as
        # in the oracle, so the fold is pinned ray by ray
        "c1_m38_nofma": (scalarize(S.echelle()), c1, (38, 1), 40),
        "c1_m52_nofma": (scalarize(S.echelle()), c1, (52, 1), 40),
    }


# The reference build each case runs through (oracle/_ref/harness_<kind>):
# refgpu is the cuda_engine built for sm_100a with its own flags (FMA
# contraction on, as nvcc defaults), refgpu_nofma the same sources with
# --fmad=false.
HARNESS = {"c1_m38_nofma": "refgpu_nofma", "c1_m52_nofma": "refgpu_nofma"}


def spec_arrays(specs):
    """Scheme as plain arrays (for the fixture file)."""
    rows = []
    for s in specs:
        p = list(s.params) + [0.0] * (16 - len(s.params))
        rows.append([s.cls, s.type, s.shape, s.grating_type, s.order, s.gr_const, len(s.params)] + p +
                    list(s.size) + list(s.center) + list(s.distance) + list(s.angles) +
                    [float(s.n1), float(s.n2)])
    return np.array(rows, dtype=np.float64)


def main(out_dir=HERE, only=None):
    os.makedirs(out_dir, exist_ok=True)
    for name, (specs, kw, orders, n_per) in cases().items():
        if only and name not in only:
            continue
        kind = HARNESS.get(name, "refgpu")
        if H.harness(kind) is None:
            raise SystemExit(f"oracle/_ref/harness_{kind} is not built")
        beam = S.make_beam(0, n_per, kw["n_lambda"], kw["radius"], kw["lam_range"], 20141203, orders=orders)
        rays = O.generate([beam], beam.n_rays)
        if name.endswith("_tagged"):
            # mirrors only: the wavelength is free, so it carries the ray index
            rays.lambda_[:] = 0.4 + 1e-7 * np.arange(rays.n)
        rc, out = H.run_trace(kind, specs, list(orders), rays)
        inp = np.stack([rays.X, rays.Y, rays.Z, rays.cX, rays.cY, rays.cZ, rays.lambda_])
        payload = dict(rc=rc, input=inp, scheme=spec_arrays(specs), orders=np.array(orders, dtype=np.int64))
        if out is not None:
            n, ng, nl, state = out
            payload.update(n=n, n_good=ng, output=state)
        np.savez_compressed(os.path.join(out_dir, f"{name}.npz"), **payload)
        print(name, "rc", rc, "n_good", payload.get("n_good"), flush=True)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = [a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")]
    main(args[0] if args else HERE, only=[o for x in only for o in x.split(",")] or None)
