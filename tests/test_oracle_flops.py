"""The op-counting oracle (oracle/flop_count.hpp) and the algorithmic FLOP
table of the benchmark scheme (rt_b200/data/flops_c1.json) -- CPU tests.

The oracle's per-ray functions are templates on the scalar type; on the
counting scalar they count the reference algorithm's add, subtract,
multiply, divide and square-root operations while taking exactly the FP64
oracle's branches.  Known answers by hand for one-surface schemes, and the
committed table reproduced from the oracle.
"""
import json
import os

import numpy as np

import pyoracle as O
from rt_b200 import ffi, schemes as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _one_surface(spec, n=10):
    b = [S.make_beam(0, n, 1, 5.0, (0.5, 0.5), 1)]
    rays = O.generate(b, n)
    ops, reached = O.count_flops(S.to_c([spec], O.spline_init).surfaces, b, rays)
    return ops, reached, n


def test_hand_counted_surfaces():
    # translation 3, Normalize 13 (three products, four quotients, two sums,
    # one square root, one product; then three quotients), plane root 5
    # (s0 = -Z/cZ; X += cX s0; Y += cY s0), circular aperture 5 (xr, yr, xr^2 + yr^2;
    # R^2 once per surface), plane mirror 0 (cZ = -cZ), Normalize 13
    mirror = S.SurfaceSpec(ffi.PLANE, ffi.MIRROR, shape=ffi.CIRCLE, size=(1000.0, 0.0), distance=(0.0, 0.0, 100.0))
    ops, reached, n = _one_surface(mirror)
    assert reached[0] == n and ops[0] == n * (3 + 13 + 5 + 5 + 0 + 13)
    # a rectangle computes xr, yr and four bounds centre +- size / 2 per ray
    # (surface.cpp:287-305): 10
    det = S.SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(1000.0, 1000.0),
                        distance=(0.0, 0.0, 100.0))
    ops, _, n = _one_surface(det)
    assert ops[0] == n * (3 + 13 + 5 + 10 + 13)


def test_committed_table_is_the_oracles():
    import importlib.util
    spec = importlib.util.spec_from_file_location("count_flops", os.path.join(ROOT, "oracle", "count_flops.py"))
    cf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cf)
    committed = json.load(open(os.path.join(ROOT, "rt_b200", "data", "flops_c1.json")))
    fresh = cf.table(committed["sample_rays"] // (len(S.C1_ORDERS) * S.C1_NLAMBDA))
    assert fresh["sample_rays"] == committed["sample_rays"]
    for a, b in zip(fresh["surfaces"], committed["surfaces"]):
        assert a["rays_reaching"] == b["rays_reaching"]
        assert abs(a["ops_per_ray"] - b["ops_per_ray"]) <= 1e-9 * b["ops_per_ray"]
    assert fresh["lost_ray_renormalize_ops"] == committed["lost_ray_renormalize_ops"]
    # surfaces without iterations cost the same for every ray
    for row in committed["surfaces"][:2]:
        assert row["ops_per_ray"] == int(row["ops_per_ray"])
