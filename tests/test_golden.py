"""Pins of the CPU oracle to the reference CUDA engine (no GPU needed).

tests/golden/*.npz hold inputs and outputs of the reference's own host
classes over its own cuda_engine (built for sm_100a, run on a B200 by
tests/golden/make_golden.py).  The reference build contracts multiply-adds
into FMAs, the oracle does not, so values are compared within the parity
tolerances (positions 1e-9 mm, direction cosines 1e-12) and flags, counts
and wavelengths exactly.

Schemes with a toric surface are compared ray by ray only where the rays can
be identified (mirrors_tagged: the wavelength carries the ray index), or
where the reference ran without FMA contraction (the *_nofma cases, C1's
toric fold): the reference's toric iteration divides 0/0 for rays that
converge exactly (rt_cuda_engine_surface.cu:390), which rays do depends on
FMA contraction, and Beam::Rearrange then orders the two outputs
differently.  Without contraction the reference rounds every operation as
the oracle does, and the *_nofma outputs equal the oracle's bit for bit.
"""
import os

import numpy as np
import pytest

import pyoracle as O
from rt_b200 import schemes as S

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

import sys  # noqa: E402
sys.path.insert(0, GOLDEN)
import make_golden as G  # noqa: E402

CASES = G.cases()
POS_TOL, COS_TOL = 1e-9, 1e-12


def _load(name):
    p = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(p):
        pytest.skip(f"fixture {name} not generated")
    return np.load(p)


def _run(name, d):
    specs, kw, orders, n_per = CASES[name]
    assert np.array_equal(G.spec_arrays(specs), d["scheme"]), "scheme drifted from the fixture"
    beam = S.make_beam(0, n_per, kw["n_lambda"], kw["radius"], kw["lam_range"], 20141203, orders=orders)
    rays = O.HostRays(beam.n_rays)
    for i, f in enumerate(O.HostRays.FIELDS):
        getattr(rays, f)[:] = d["input"][i]
    cs = S.to_c(specs, O.spline_init)
    st, ng = O.trace_literal(cs.surfaces, beam, rays)
    return st, ng, np.stack([getattr(rays, f) for f in O.HostRays.FIELDS])


@pytest.mark.parametrize("name", [n for n in CASES if n not in ("c1_m38", "c1_m52", "mirrors", "mirrors_tagged")])
def test_oracle_matches_reference_engine(name):
    d = _load(name)
    st, ng, ours = _run(name, d)
    assert st == int(d["rc"])
    if st != 0:
        return
    ref = d["output"]
    assert ng == int(d["n_good"])
    assert np.array_equal(ours[6], ref[6]), "wavelengths (ray order) differ"
    assert np.array_equal(np.isnan(ours), np.isnan(ref))
    fin = ~np.isnan(ref)
    assert np.all(np.abs(ours[:3] - ref[:3])[fin[:3]] <= POS_TOL)
    assert np.all(np.abs(ours[3:6] - ref[3:6])[fin[3:6]] <= COS_TOL)
    if G.HARNESS.get(name) == "refgpu_nofma":
        assert np.array_equal(ours[fin], ref[fin]), "the reference without FMA contraction differs in bits"


def test_toric_rays_match_by_tag():
    """Rays identified by their wavelength tag: every ray that stays finite in
    both engines has the same fate and, if good, the same state."""
    d = _load("mirrors_tagged")
    st, ng, ours = _run("mirrors_tagged", d)
    assert st == int(d["rc"]) == 0
    ref = d["output"]
    n = ref.shape[1]
    n_good_ref = int(d["n_good"])
    tag = lambda lam: np.rint((lam - 0.4) / 1e-7).astype(np.int64)
    ours_by = np.empty_like(ours)
    ref_by = np.empty_like(ref)
    ours_by[:, tag(ours[6])] = ours
    ref_by[:, tag(ref[6])] = ref
    good_ours = np.zeros(n, bool)
    good_ours[tag(ours[6][:ng])] = True
    good_ref = np.zeros(n, bool)
    good_ref[tag(ref[6][:n_good_ref])] = True
    finite = np.isfinite(ours_by).all(0) & np.isfinite(ref_by).all(0)
    assert finite.mean() > 0.5
    assert np.array_equal(good_ours[finite], good_ref[finite])
    both = finite & good_ours
    assert np.all(np.abs(ours_by[:3, both] - ref_by[:3, both]) <= POS_TOL)
    assert np.all(np.abs(ours_by[3:6, both] - ref_by[3:6, both]) <= COS_TOL)


@pytest.mark.parametrize("name", ["c1_m38", "c1_m52", "mirrors"])
def test_toric_schemes_agree_in_aggregate(name):
    d = _load(name)
    st, ng, ours = _run(name, d)
    assert st == int(d["rc"])
    if st == 0:
        ref = d["output"]
        assert abs(ng - int(d["n_good"])) <= 0.25 * ref.shape[1]
        assert np.array_equal(np.sort(ours[6]), np.sort(ref[6]))
