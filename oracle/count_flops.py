"""Writes the algorithmic FLOP table of the benchmark scheme.

TEST INFRASTRUCTURE: runs the CPU oracle's per-ray functions on the counting
scalar of flop_count.hpp (add, subtract, multiply, divide, square root 1
each) over a seeded sample of C1's rays -- every echelle order, every
wavelength -- with the benchmark's quirk fixes, and stores per surface the
operations per ray that reaches it.  The table is the reference algorithm's
work: bench.py multiplies it by the rays each surface receives in a run.

  python oracle/count_flops.py [out.json] [rays_per_lambda]
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [ROOT, HERE]

import pyoracle as O  # noqa: E402
from rt_b200 import schemes as S  # noqa: E402

FIXES = 3  # the benchmark's toric fixes (bench.py)


def table(n_per_lambda: int = 200) -> dict:
    specs = S.echelle()
    beams = S.c1_beams(n_per_lambda=n_per_lambda)
    n = S.total_rays(beams)
    rays = O.generate(beams, n)
    cs = S.to_c(specs, O.spline_init)
    ops, reached = O.count_flops(cs.surfaces, beams, rays, fixes=FIXES)
    rows = []
    for k, s in enumerate(specs):
        rows.append({"surface": k, "comment": s.comment, "rays_reaching": int(reached[k]),
                     "ops_per_ray": float(ops[k]) / max(1, int(reached[k]))})
    return {"scheme": "C1 cross-dispersed echelle", "fixes": FIXES, "sample_rays": n,
            "counting": "add, subtract, multiply, divide, square root = 1; comparisons, negation, fabs = 0; "
                        "per ray reaching the surface: its transform, Normalize, intersection (iterations "
                        "included), aperture test, action and Normalize",
            "surfaces": rows, "lost_ray_renormalize_ops": int(ops[len(specs)]),
            "ops_per_input_ray": float(ops.sum()) / n}


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "rt_b200", "data", "flops_c1.json")
    npl = int(sys.argv[2]) if len(sys.argv) > 2 else 200
    t = table(npl)
    with open(out, "w") as f:
        json.dump(t, f, indent=1)
        f.write("\n")
    print(json.dumps(t, indent=1))
