"""The reverse sweep of rtb_adjoint_backward against the forward-mode passes
(RTB_ADJOINT_BACKWARD=passes) and the forward-mode sensitivities (GPU tests).

Both compute the derivative of the same expressions: the reverse sweep as
the transpose of each stage's Jacobian, the passes with dual numbers.  So the
gradients agree to rounding:
* C4's spot-merit gradient (24 parameters, 1e7 rays' worth of C4 at a
  smaller ray count) to 1e-12 relative per parameter;
* on the coverage schemes -- every intersection kind, action and grating
  type, in the reference's quirk mode and with the toric fixes -- with every
  parameter their surfaces admit and random per-ray seeds: against the passes
  and against the contraction of jvp, to 1e-12 of the sum of the rays'
  absolute contributions.
"""
import numpy as np
import pytest
import torch

from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu


def _backward(adj, gX, gY, monkeypatch, passes):
    if passes:
        monkeypatch.setenv("RTB_ADJOINT_BACKWARD", "passes")
    else:
        monkeypatch.delenv("RTB_ADJOINT_BACKWARD", raising=False)
    return adj.backward(gX, gY)


def test_c4_merit_gradient_reverse_equals_passes(monkeypatch):
    beams = S.c4_beams(n_per_lambda=4000)
    n = S.total_rays(beams)
    cs = S.to_c(S.littrow_free_asphere(), E.spline_init)
    rays = E.generate(beams, n)
    adj = E.Adjoint(cs.surfaces, S.c4_params(), beams, n, fixes=ffi.FIX_ASPHERE_ROOT)
    st, _ = adj.forward(None, rays)
    assert st == ffi.OK
    lam = np.linspace(S.C4_LAMBDA[0], S.C4_LAMBDA[1], S.C4_NLAMBDA)
    _, gX, gY = adj.spot_merit(S.c4_target_x(lam), 10.0)
    g_rev = _backward(adj, gX, gY, monkeypatch, False)
    g_pas = _backward(adj, gX, gY, monkeypatch, True)
    rel = np.abs(g_rev - g_pas) / np.abs(g_pas)
    print("C4 merit gradient: reverse vs passes, max rel", rel.max())
    assert rel.max() <= 1e-12, (int(np.argmax(rel)), rel.max())
    assert np.array_equal(g_rev, _backward(adj, gX, gY, monkeypatch, False))  # reproducible
    adj.destroy()


def all_params(specs, limit=ffi.ADJ_MAX_PARAMS):
    """Every parameter the surfaces admit (rtb_adjoint_create's rules): shape
    parameters first, then distances and angles, at most `limit`."""
    shape, geo = [], []
    for k, sp in enumerate(specs):
        curved = sp.cls in (ffi.CONIC, ffi.TORIC)
        if curved and sp.params[0] != 0.0:
            shape.append((k, ffi.PARAM_CURVATURE, 0))
        if (sp.cls == ffi.CONIC and sp.params[1] != -1.0) or sp.cls == ffi.TORIC:
            shape.append((k, ffi.PARAM_CONIC, 0))
        if curved:
            shape += [(k, ffi.PARAM_POLY, i) for i in range(int(sp.params[2]))]
        if sp.cls == ffi.TORIC:
            shape.append((k, ffi.PARAM_TORIC_CR, 0))
        if sp.type == ffi.GRATING:
            shape.append((k, ffi.PARAM_GROOVE_DENSITY, 0))
        geo += [(k, ffi.PARAM_DISTANCE, i) for i in range(3)] + [(k, ffi.PARAM_ANGLE, i) for i in range(3)]
    return (shape + geo)[:limit]


@pytest.mark.parametrize("fixes", [0, ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP | ffi.FIX_ASPHERE_ROOT])
@pytest.mark.parametrize("name", ["mirrors", "lenses", "gratings"])
def test_reverse_equals_passes_and_jvp_on_every_kind(name, fixes, monkeypatch):
    specs = S.coverage_schemes()[name]
    beams = [S.make_beam(0, 400, 5, 10.0, (0.4, 0.8), 17)]
    n = S.total_rays(beams)
    cs = S.to_c(specs, E.spline_init)
    params = all_params(specs)
    rays = E.generate(beams, n)
    adj = E.Adjoint(cs.surfaces, params, beams, n, fixes=fixes)
    st, stats = adj.forward(None, rays)
    assert st == ffi.OK and stats.n_good > n // 10
    gen = torch.Generator(device="cuda").manual_seed(11)
    gX = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    gY = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    # in the quirk mode the toric 0/0 gives some rays NaN positions that pass
    # the apertures after it (NaN compares false): no seed on those
    finite = torch.isfinite(adj.X) & torch.isfinite(adj.Y)
    gX, gY = torch.where(finite, gX, 0.0), torch.where(finite, gY, 0.0)
    g_rev = _backward(adj, gX, gY, monkeypatch, False)
    g_pas = _backward(adj, gX, gY, monkeypatch, True)
    P = len(params)
    worst = 0.0
    for j in range(P):
        e = np.zeros(P)
        e[j] = 1.0
        dX, dY = adj.jvp(e)
        contrib = torch.where(finite, gX * dX + gY * dY, 0.0)
        scale = float(contrib.abs().sum())
        dot = float(contrib.sum())
        tol = 1e-12 * scale + 1e-300
        err = max(abs(g_rev[j] - g_pas[j]), abs(g_rev[j] - dot))
        worst = max(worst, err / (scale + 1e-300))
        assert err <= tol, (params[j], g_rev[j], g_pas[j], dot, scale)
    print(name, fixes, P, "parameters, worst error / sum |contributions|:", worst)
    adj.destroy()


@pytest.mark.parametrize("name", ["c4", "mirrors", "lenses", "gratings"])
def test_reverse_sweep_compiled_for_the_scheme_equals_generic(name, monkeypatch):
    """rtb_adjoint_create compiles the forward, the reverse sweep and the
    sensitivities for the scheme's structure (RTB_SPECIALIZE=0: the generic
    kernels); both run the same IEEE operations in the same order: the same
    positions, gradient and sensitivity bits, also with
    the parameters moved off their create-time values (angles and distances
    away from zero change which transforms apply, which the compiled kernel
    reads at run time)."""
    if name == "c4":
        specs, params, fixes = S.littrow_free_asphere(), S.c4_params(), ffi.FIX_ASPHERE_ROOT
    else:
        specs = S.coverage_schemes()[name]
        params, fixes = all_params(specs), ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP
    beams = [S.make_beam(0, 400, 5, 10.0, (0.4, 0.8), 23)]
    n = S.total_rays(beams)
    cs = S.to_c(specs, E.spline_init)
    rays = E.generate(beams, n)
    grads = []
    for spec in ("1", "0"):
        monkeypatch.setenv("RTB_SPECIALIZE", spec)
        adj = E.Adjoint(cs.surfaces, params, beams, n, fixes=fixes)
        theta = adj.theta()
        out = []
        for move in (0.0, 1e-3):
            th = theta + move * np.where(np.arange(len(theta)) % 2 == 0, 1.0, -1.0) * np.maximum(np.abs(theta), 1.0)
            if move:
                # groove densities stay positive; everything else moves by 1e-3 (relative, or absolute at 0)
                th = np.where(theta > 0, np.maximum(th, 0.5 * theta), th)
            st, _ = adj.forward(th, rays)
            assert st == ffi.OK
            out.append((adj.X.clone(), adj.Y.clone(), adj.flag.clone()))
            gen = torch.Generator(device="cuda").manual_seed(3)
            gX = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
            gY = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
            finite = torch.isfinite(adj.X) & torch.isfinite(adj.Y)
            gX, gY = torch.where(finite, gX, 0.0), torch.where(finite, gY, 0.0)
            monkeypatch.delenv("RTB_ADJOINT_BACKWARD", raising=False)
            out.append(adj.backward(gX, gY))
            d = np.random.default_rng(7).normal(size=len(theta))
            dX, dY = adj.jvp(d)
            out.append((dX.clone(), dY.clone()))
        grads.append(out)
        adj.destroy()
    for a, b in zip(*grads):
        if isinstance(a, tuple) and len(a) == 3:  # the forward's outputs
            assert torch.equal(a[2], b[2])
            g = a[2] == 1
            assert torch.equal(a[0][g].view(torch.int64), b[0][g].view(torch.int64))
            assert torch.equal(a[1][g].view(torch.int64), b[1][g].view(torch.int64))
        elif isinstance(a, tuple):  # the sensitivities along one direction
            for x, y in zip(a, b):
                assert torch.equal(torch.nan_to_num(x).view(torch.int64), torch.nan_to_num(y).view(torch.int64))
        else:
            assert np.array_equal(a, b), np.max(np.abs(a - b))
