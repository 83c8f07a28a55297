"""Throughput-curve cases (Scheme::ComputeQE) shared by the QE tests and the
fixture generator: QE surfaces of the benchmark schemes, wavelength-range
rows and numbers of wavelengths.

Each case is (specs, rows, n_lambda): specs are SurfaceSpec of the QE
surfaces in scheme order (qe_curve, gratings with order, const, alpha,
gamma, blaze_angle, rule_params), rows the ranges "w1 w2 [order per
grating]" as a scheme's range attribute or range file gives them.
"""
from __future__ import annotations

import math

from rt_b200 import ffi, schemes as S


def tolerance(case: str) -> float:
    """Agreement, relative to each curve's largest value, of curves whose
    blaze function runs on different sin, cos and asin (host libm against
    the GPU's).  The blaze normalisation sums I1 over every propagating
    order.  For a coarse grating (the echelle, 79 l/mm: eps / lambda > 20,
    dozens of orders) some order's diffracted angle beta comes within 1e-4
    rad of c - 90 deg (the facet's grazing direction), where
    U = pi eps / lambda cos(beta) / cos(c - beta) (...) reaches 1e6 and one
    ulp of beta moves sin(U) by ~1e-7: the reference's own curve carries
    that noise (measured: up to 5e-9 of the curve's maximum between the
    host's libm and the reference's kernel).  With few orders the curves
    agree to rounding (measured: 4e-15)."""
    return 1e-8 if case.startswith("c1") or case == "orders_and_angles" else 1e-12


def qe_specs(specs):
    return [s for s in specs if s.cls != ffi.AUX_CLASS and s.type in S.QE_TYPES]


def scalar_qe(specs, value=0.8):
    """The same surfaces with every tabulated qe_curve replaced by a single
    value: the reference's spline_init kernel runs the spline recurrence in
    parallel (rt_cuda_engine_spline.cu:21-37), so curves from tables through
    the reference's CUDA engine are not reproducible."""
    out = []
    for s in specs:
        s = S.SurfaceSpec(**s.__dict__)
        if not isinstance(s.qe, (int, float)):
            s.qe = value
        out.append(s)
    return out


def grating(order, gr_const, alpha, gamma, blaze, rule=(), qe=0.9):
    return S.SurfaceSpec(ffi.PLANE, ffi.GRATING, order=order, gr_const=gr_const, alpha=alpha, gamma=gamma,
                         blaze=blaze, rule_params=rule, qe=qe)


def blaze_rows(m_lo=64, m_hi=150, step=6, cross_order=1):
    """Echelle orders around their blaze peaks: order m over lambda_B(m) (1 +- 1/m),
    lambda_B = 2 d sin(63.5 deg) cos(4 deg) / m for the C1 echelle."""
    d = 1000.0 / 31.6
    rows = []
    for m in range(m_lo, m_hi + 1, step):
        lb = 2 * d * math.sin(math.radians(63.5)) * math.cos(math.radians(4.0)) / m
        rows.append([lb * (1 - 1.0 / m), lb * (1 + 1.0 / m), m, cross_order])
    return rows


def cases() -> dict:
    c0 = qe_specs(S.littrow_free())
    c1 = qe_specs(S.echelle())
    c4 = qe_specs(S.littrow_free_asphere())
    out = {
        "c0": (c0, [list(S.C0_LAMBDA)], 301),
        "c4": (c4, [list(S.C4_LAMBDA)], 64),
        # the C1 range file: one row per echelle order over the full range
        "c1_ranges": (c1, [[S.C1_LAMBDA[0], S.C1_LAMBDA[1], m, 1] for m in S.C1_ORDERS], 129),
        "c1_blaze": (c1, blaze_rows(), 257),
        # one range with orders in the row: the orders come from the gratings
        "c1_one_range": (c1, [[0.45, 0.47, 120, 2]], 65),
    }
    rules = [grating(1, 1.0 / 0.6, 10.0, 0.0, 9.5, rule=r) for r in
             [(), (0.25,), (0.1, 0.6), (-0.5, 1.5), (0.3, 0.9, 0.5)]]
    out["rule_params"] = (rules, [[0.4, 0.7]], 101)
    out["orders_and_angles"] = ([grating(-2, 1000.0 / 600.0, 25.0, 3.0, 21.0, qe=0.7),
                                 grating(3, 1000.0 / 79.0, 40.0, 10.0, 44.0, rule=(0.05, 0.95), qe=0.95),
                                 S.SurfaceSpec(ffi.PLANE, ffi.DETECTOR, qe=0.6)], [[0.42, 0.61]], 97)
    # order 2 of 1200 l/mm stops propagating at 0.587 um: the blaze function's
    # asin is taken of a value > 1 and the reference's curve is NaN there
    out["evanescent"] = ([grating(2, 1000.0 / 1200.0, 25.0, 0.0, 26.7)], [[0.42, 0.61]], 97)
    return out
