"""Result files for the losses_comp / print_lambda tests: the CPU oracle's
literal replica of Scheme::run traces a beam and the result is written as
Beam::Save writes it (beam.cpp:636-715: size_t n, n_good, n_lambda, then X Y
Z cX cY cZ lambda of the good rays, then of the lost rays)."""
from __future__ import annotations

import os

import numpy as np

import pyoracle as O
from rt_b200 import schemes as S

FIELDS = ("X", "Y", "Z", "cX", "cY", "cZ", "lambda_")


def write_dat(path: str, rays, n_good: int, n_lambda: int) -> None:
    with open(path, "wb") as f:
        f.write(np.array([rays.n, n_good, n_lambda], dtype=np.uint64).tobytes())
        for part in (slice(0, n_good), slice(n_good, rays.n)):
            for name in FIELDS:
                f.write(np.ascontiguousarray(getattr(rays, name)[part], dtype=np.float64).tobytes())


def read_lambda(path: str):
    """(n, n_good, n_lambda, lambda of all rays, good first)."""
    with open(path, "rb") as f:
        n, ng, nl = (int(v) for v in np.frombuffer(f.read(24), dtype=np.uint64))
        good = np.frombuffer(f.read(7 * ng * 8), dtype=np.float64).reshape(7, ng)[6]
        bad = np.frombuffer(f.read(7 * (n - ng) * 8), dtype=np.float64).reshape(7, n - ng)[6]
    return n, ng, nl, np.concatenate([good, bad])


def traced(specs, n_per: int, n_lambda: int, radius: float, lam, seed: int, orders=()):
    beam = S.make_beam(0, n_per, n_lambda, radius, lam, seed, orders=orders)
    rays = O.generate([beam], beam.n_rays)
    cs = S.to_c(specs, O.spline_init)
    st, ng = O.trace_literal(cs.surfaces, beam, rays)
    return rays, ng


def cases() -> dict:
    """name -> (specs, n_per_lambda, n_lambda, radius, range, seed, orders)."""
    return {
        "c0": (S.littrow_free(), 2000, S.C0_NLAMBDA, S.C0_RADIUS, S.C0_LAMBDA, S.SEED, ()),
        "c1_m38": (S.echelle(), 300, S.C1_NLAMBDA, S.C1_RADIUS, S.C1_LAMBDA, S.SEED + 38, (38, 1)),
        "c1_m52": (S.echelle(), 300, S.C1_NLAMBDA, S.C1_RADIUS, S.C1_LAMBDA, S.SEED + 52, (52, 1)),
        "c0_mono": (S.littrow_free(), 3000, 1, S.C0_RADIUS, (0.55, 0.55), S.SEED + 1, ()),
    }


def write_case(d: str, name: str) -> str:
    specs, npl, nl, radius, lam, seed, orders = cases()[name]
    rays, ng = traced(specs, npl, nl, radius, lam, seed, orders)
    path = os.path.join(d, f"{name}.dat")
    write_dat(path, rays, ng, nl)
    return path


def write_synthetic(path: str, n_lambda: int, nl: int, seed: int, lam0=0.38, lam1=0.9) -> None:
    """A result file of n_lambda wavelengths x nl rays (composite layout),
    each wavelength losing a random share of its rays except the longest,
    which keeps all of them: then no window of losses_comp's count runs past
    the good rays (where the reference reads beyond its array, and its result
    depends on what lies there)."""
    rng = np.random.default_rng(seed)
    grid = lam0 + (lam1 - lam0) / (n_lambda - 1) * np.arange(n_lambda) if n_lambda > 1 else np.array([lam0])
    lam = np.tile(grid, nl)
    keep = rng.uniform(size=lam.size) < rng.uniform(0.05, 0.95, size=n_lambda)[np.tile(np.arange(n_lambda), nl)]
    keep |= lam == grid[-1]
    order = np.concatenate([rng.permutation(np.nonzero(keep)[0]), rng.permutation(np.nonzero(~keep)[0])])

    class R:
        pass
    r = R()
    r.n = lam.size
    for name in FIELDS:
        setattr(r, name, rng.normal(size=lam.size) if name != "lambda_" else lam[order])
    write_dat(path, r, int(keep.sum()), n_lambda)
