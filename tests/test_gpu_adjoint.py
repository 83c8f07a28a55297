"""Adjoint gradients (rtb_adjoint_*) on C4: C0's spectrograph extended with
an even-asphere field flattener, 64 wavelengths over 0.40-0.70 um, 24
parameters (GPU tests).

* The forward is the plain FP64 engine: the same bits as rtb_trace's fused
  FP64 trace, also with the parameters moved.
* The backward (reverse sweep over the surfaces, and inside each surface,
  from checkpoints) equals the contraction of the forward-mode sensitivities
  with the same seeds.
* Forward-mode sensitivities match central finite differences ray by ray.
* The merit sum_lambda RMS + 10 (xbar - x_t(lambda))^2, differentiated
  through a torch.autograd.Function around forward/backward, matches central
  finite differences of the FP64 forward (relative step 1e-6) to 1e-6.
"""
import numpy as np
import pytest
import torch

from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu

WEIGHT = 10.0
REL_STEP = 1e-6
# the reference's asphere iteration reports the point before its last Newton
# update (up to 1e-7 mm short of the root), which makes the forward jump when a
# parameter moves the stopping decision; the gradient is of the converged model
FIXES = ffi.FIX_ASPHERE_ROOT


def setup(n_per_lambda=1600):
    specs = S.littrow_free_asphere()
    cs = S.to_c(specs, E.spline_init)
    beams = S.c4_beams(n_per_lambda=n_per_lambda)
    n = S.total_rays(beams)
    rays = E.generate(beams, n)
    torch.cuda.synchronize()
    adj = E.Adjoint(cs.surfaces, S.c4_params(), beams, n, fixes=FIXES)
    return specs, cs, beams, n, rays, adj


def steps(theta):
    return np.where(theta != 0.0, REL_STEP * np.abs(theta), REL_STEP)


def group_ids(n, n_lambda=S.C4_NLAMBDA):
    return torch.arange(n, device="cuda") % n_lambda


def merit_difference(Xp, Yp, Xm, Ym, mask, G, target):
    """M(+) - M(-) for two forwards on the same rays, summed from per-ray
    differences (Xp - Xm is exact for nearby doubles), so that the finite
    difference keeps its digits where M itself is ~1e5 times larger.
    Rays are grouped by wavelength index i mod G (n = G * rays per group)."""
    Xp, Yp, Xm, Ym = (torch.where(mask, a, torch.zeros_like(a)) for a in (Xp, Yp, Xm, Ym))
    w = mask.double().view(-1, G)
    N = w.sum(0)
    mean = lambda a: (a.view(-1, G) * w).sum(0) / N  # noqa: E731
    Dx, Dy = mean(Xp - Xm), mean(Yp - Ym)              # xbar+ - xbar-
    Sx, Sy = mean(Xp + Xm), mean(Yp + Ym)              # xbar+ + xbar-
    up, um = Xp.view(-1, G) - (Sx + Dx) / 2, Xm.view(-1, G) - (Sx - Dx) / 2
    vp, vm = Yp.view(-1, G) - (Sy + Dy) / 2, Ym.view(-1, G) - (Sy - Dy) / 2
    d_du = (Xp - Xm).view(-1, G) - Dx                  # u+ - u-, accurate
    d_dv = (Yp - Ym).view(-1, G) - Dy
    drms2 = ((d_du * (up + um) + d_dv * (vp + vm)) * w).sum(0) / N
    rms_p = torch.sqrt(((up * up + vp * vp) * w).sum(0) / N)
    rms_m = torch.sqrt(((um * um + vm * vm) * w).sum(0) / N)
    return float((drms2 / (rms_p + rms_m)).sum() + WEIGHT * (Dx * (Sx - 2 * target)).sum())


def merit_torch(X, Y, mask, gid, target, G):
    X, Y = torch.where(mask, X, torch.zeros_like(X)), torch.where(mask, Y, torch.zeros_like(Y))
    w = mask.double()
    N = torch.zeros(G, dtype=torch.float64, device="cuda").index_add_(0, gid, w)
    xbar = torch.zeros(G, dtype=torch.float64, device="cuda").index_add_(0, gid, X * w) / N
    ybar = torch.zeros(G, dtype=torch.float64, device="cuda").index_add_(0, gid, Y * w) / N
    d2 = ((X - xbar[gid]) ** 2 + (Y - ybar[gid]) ** 2) * w
    rms = torch.sqrt(torch.zeros(G, dtype=torch.float64, device="cuda").index_add_(0, gid, d2) / N)
    return (rms + WEIGHT * (xbar - target) ** 2).sum()


class TraceFn(torch.autograd.Function):
    """The shape rtb_adjoint_forward / rtb_adjoint_backward are made for."""

    @staticmethod
    def forward(ctx, theta, adj, rays):
        st, _ = adj.forward(theta.detach().cpu().numpy(), rays)
        assert st == ffi.OK
        ctx.adj = adj
        return adj.X.clone(), adj.Y.clone()

    @staticmethod
    def backward(ctx, gX, gY):
        g = ctx.adj.backward(gX.contiguous(), gY.contiguous())
        return torch.as_tensor(g, dtype=torch.float64), None, None


def test_forward_equals_plain_fp64_engine():
    specs, cs, beams, n, rays, adj = setup()
    st, stats = adj.forward(None, rays)
    ref = rays.copy()
    st2, stats2 = E.trace(cs.surfaces, beams, ref, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, fixes=FIXES))
    assert st == st2 == ffi.OK and stats.n_good == stats2.n_good and stats.ray_surfaces == stats2.ray_surfaces
    assert torch.equal(adj.flag, ref.flag)
    g = ref.flag == 1
    assert torch.equal(adj.X[g].view(torch.int64), ref.X[g].view(torch.int64))
    assert torch.equal(adj.Y[g].view(torch.int64), ref.Y[g].view(torch.int64))
    # with every parameter moved: the plain engine on the moved scheme
    theta = adj.theta()
    moved = theta + steps(theta) * 1e3 * np.where(np.arange(len(theta)) % 2 == 0, 1.0, -1.0)
    st, _ = adj.forward(moved, rays)
    specs2 = [S.SurfaceSpec(**s.__dict__) for s in specs]
    for (k, kind, idx), v in zip(S.c4_params(), moved):
        sp = specs2[k]
        if kind == ffi.PARAM_CURVATURE:
            sp.params = (v, *sp.params[1:])
        elif kind == ffi.PARAM_CONIC:
            sp.params = (sp.params[0], v, *sp.params[2:])
        elif kind == ffi.PARAM_POLY:
            p = list(sp.params)
            p[3 + idx] = v
            sp.params = tuple(p)
        elif kind == ffi.PARAM_DISTANCE:
            d = list(sp.distance)
            d[idx] = v
            sp.distance = d
        elif kind == ffi.PARAM_ANGLE:
            a = list(sp.angles)
            a[idx] = v
            sp.angles = a
        elif kind == ffi.PARAM_GROOVE_DENSITY:
            sp.gr_const = 1000.0 / v
    cs2 = S.to_c(specs2, E.spline_init)
    ref = rays.copy()
    st2, _ = E.trace(cs2.surfaces, beams, ref, E.opts(engine=ffi.ENGINE_FUSED, precision=ffi.FP64, fixes=FIXES))
    assert st == st2 == ffi.OK
    assert torch.equal(adj.flag, ref.flag)
    g = ref.flag == 1
    assert torch.equal(adj.X[g], ref.X[g]) and torch.equal(adj.Y[g], ref.Y[g])
    adj.destroy()


def test_backward_equals_forward_mode_contraction():
    _, _, _, n, rays, adj = setup()
    adj.forward(None, rays)
    gen = torch.Generator(device="cuda").manual_seed(5)
    gX = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    gY = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    grad = adj.backward(gX, gY)
    P = len(grad)
    for j in range(P):
        e = np.zeros(P)
        e[j] = 1.0
        dX, dY = adj.jvp(e)
        dot = float((gX * dX + gY * dY).sum())
        assert abs(grad[j] - dot) <= 1e-10 * max(abs(dot), 1e-300) + 1e-300, (j, grad[j], dot)
    # reproducible
    assert np.array_equal(grad, adj.backward(gX, gY))
    adj.destroy()


def test_forward_mode_matches_central_differences_per_ray():
    _, _, _, n, rays, adj = setup(n_per_lambda=400)
    adj.forward(None, rays)
    theta = adj.theta()
    base_flag = adj.flag.clone()
    h = steps(theta)
    worst = []
    for j in range(len(theta)):
        e = np.zeros(len(theta))
        e[j] = 1.0
        dX, dY = adj.jvp(e)
        out = []
        for sgn in (1.0, -1.0):
            adj.forward(theta + sgn * h[j] * e, rays)
            out.append((adj.X.clone(), adj.Y.clone(), adj.flag.clone()))
        adj.forward(None, rays)
        m = (base_flag == 1) & (out[0][2] == 1) & (out[1][2] == 1)
        fx = (out[0][0] - out[1][0]) / (2 * h[j])
        fy = (out[0][1] - out[1][1]) / (2 * h[j])
        # a central difference of a forward rounded to ~1e-13 of |X| carries
        # an error of about 1e-13 |X| / h: allow that on top of 1e-6 relative
        floor = 1e-13 * (adj.X.abs() + adj.Y.abs() + 1.0) / h[j]
        err = torch.hypot(fx - dX, fy - dY)
        tol = 1e-6 * torch.hypot(dX, dY) + floor
        bad = int(((err > tol) & m).sum())
        worst.append((j, bad, int(m.sum()), float((err / tol)[m].max())))
    print(worst)
    for j, bad, nm, ratio in worst:
        assert bad <= 1e-3 * nm, (j, bad, nm, ratio)
    adj.destroy()


@pytest.mark.parametrize("n_per_lambda", [1600, 156250])
def test_merit_gradient_matches_central_differences(n_per_lambda):
    """C4 at 1e5 rays and at its full 1e7 rays."""
    _, _, beams, n, rays, adj = setup(n_per_lambda)
    theta0 = adj.theta()
    P = len(theta0)
    h = steps(theta0)
    gid = group_ids(n)
    lam = np.linspace(S.C4_LAMBDA[0], S.C4_LAMBDA[1], S.C4_NLAMBDA)
    target = torch.as_tensor(S.c4_target_x(lam), dtype=torch.float64, device="cuda")
    # the rays good at theta0 and at every finite-difference point
    adj.forward(None, rays)
    mask = adj.flag == 1
    pts = []
    for j in range(P):
        for sgn in (1.0, -1.0):
            t = theta0.copy()
            t[j] += sgn * h[j]
            st, _ = adj.forward(t, rays)
            assert st == ffi.OK
            mask &= adj.flag == 1
            pts.append((adj.X.clone(), adj.Y.clone()))
    fd = np.array([merit_difference(*pts[2 * j], *pts[2 * j + 1], mask, S.C4_NLAMBDA, target) / (2 * h[j])
                   for j in range(P)])
    del pts
    # adjoint: merit in torch on the same rays, gradient through TraceFn
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    X, Y = TraceFn.apply(theta, adj, rays)
    M = merit_torch(X, Y, mask, gid, target, S.C4_NLAMBDA)
    M.backward()
    g = theta.grad.numpy()
    rel = np.abs(g - fd) / np.abs(fd)
    print("merit", float(M), "rel err", rel.max(), list(zip(range(P), g, fd, rel)))
    assert np.all(np.abs(fd) > 0)
    assert rel.max() <= 1e-6, (int(np.argmax(rel)), rel.max())
    # the library's own merit and seeds agree with torch's on the forward's good rays
    adj.forward(None, rays)
    if bool(torch.equal(mask, adj.flag == 1)):
        m_lib, gX, gY = adj.spot_merit(S.c4_target_x(lam), WEIGHT)
        assert abs(m_lib - float(M)) <= 1e-12 * abs(float(M))
        g_lib = adj.backward(gX, gY)
        assert np.allclose(g_lib, g, rtol=1e-9, atol=0)
    adj.destroy()


def _two_beam_forward(n_lambda):
    """C4's scheme traced for two beams (n_lambda and 5 wavelengths) with rays
    outside both (before, between, after): the adjoint, the forward's X, Y
    and good flags (numpy), each wavelength group's ray indices and the mask
    of the rays outside every beam."""
    specs = S.littrow_free_asphere()
    cs = S.to_c(specs, E.spline_init)
    a = S.make_beam(100, 40, n_lambda, S.C0_RADIUS, S.C4_LAMBDA, S.SEED + 41)
    b = S.make_beam(100 + int(a.n_rays) + 77, 200, 5, S.C0_RADIUS, S.C4_LAMBDA, S.SEED + 42)
    beams = [a, b]
    n = int(b.first_ray + b.n_rays) + 50
    groups, lams = [], []
    for bm in beams:
        nl = int(bm.n_lambda) or 1
        for j in range(nl):
            groups.append(int(bm.first_ray) + j + nl * np.arange((int(bm.n_rays) - j + nl - 1) // nl))
            lams.append(bm.range[0] + j * (bm.range[1] - bm.range[0]) / max(1, nl - 1))
    outside = np.ones(n, bool)
    for idx in groups:
        outside[idx] = False
    rays = E.generate(beams, n)
    off = torch.as_tensor(outside, device="cuda")
    rays.flag[off] = 0  # rays outside the beams: lost on entry, never traced
    for f in E.FIELDS:
        getattr(rays, f)[off] = 0.0
    torch.cuda.synchronize()
    adj = E.Adjoint(cs.surfaces, S.c4_params(), beams, n, fixes=FIXES)
    st, _ = adj.forward(None, rays)
    assert st == ffi.OK
    X, Y = adj.X.cpu().numpy(), adj.Y.cpu().numpy()
    good = adj.flag.cpu().numpy() == 1
    return adj, X, Y, good, groups, np.array(lams), outside, [int(bm.n_lambda) or 1 for bm in beams]


def _check_seeds(gX, gY, rX, rY, outside):
    gX, gY = gX.cpu().numpy(), gY.cpu().numpy()
    scale = max(np.abs(rX).max(), np.abs(rY).max())
    assert np.abs(gX - rX).max() <= 1e-10 * scale and np.abs(gY - rY).max() <= 1e-10 * scale
    assert outside.sum() == 100 + 77 + 50 and not gX[outside].any() and not gY[outside].any()


@pytest.mark.parametrize("n_lambda", [64, 300])
def test_spot_merit_and_seeds_against_numpy(n_lambda):
    """rtb_adjoint_spot_merit on two beams with rays outside both: the merit
    and the per-ray seeds equal a numpy restatement of sum_groups RMS + w
    (xbar - x_t)^2 over each beam's wavelength groups, and the seeds of rays
    outside every beam are 0.  64 wavelengths take the index-order path, 300
    (more than a block's threads) the group-by-group one."""
    adj, X, Y, good, groups, _, outside, _ = _two_beam_forward(n_lambda)
    n = X.size
    target = np.linspace(-1.0, 1.0, len(groups))
    m_lib, gX, gY = adj.spot_merit(target, WEIGHT)
    M, rX, rY = 0.0, np.zeros(n), np.zeros(n)
    for g, idx in enumerate(groups):
        idx = idx[good[idx]]
        if idx.size == 0:
            continue
        xb, yb = X[idx].mean(), Y[idx].mean()
        rms = np.sqrt(np.mean((X[idx] - xb) ** 2 + (Y[idx] - yb) ** 2))
        M += rms + WEIGHT * (xb - target[g]) ** 2
        rX[idx] = (X[idx] - xb) / (idx.size * rms) + 2 * WEIGHT * (xb - target[g]) / idx.size
        rY[idx] = (Y[idx] - yb) / (idx.size * rms)
    assert abs(m_lib - M) <= 1e-12 * abs(M), (m_lib, M)
    _check_seeds(gX, gY, rX, rY, outside)
    adj.destroy()


def resolution_np(X, Y, groups, lams, nls, u):
    """The spectral-resolution merit (rtb_adjoint_resolution_merit) in numpy:
    per group, the centroid p and RMS width s of u.(X, Y); summed over the
    neighbouring wavelengths of each beam, s-bar |dlambda| / |dp| / lambda-bar.
    Also returns its derivatives in each ray's X and Y (autograd by hand)."""
    u = np.asarray(u, dtype=np.float64) / np.hypot(*u)
    q = u[0] * X + u[1] * Y
    p = np.array([q[i].mean() for i in groups])
    s = np.array([np.sqrt(np.mean((q[i] - q[i].mean()) ** 2)) for i in groups])
    M, dp, ds = 0.0, np.zeros(len(groups)), np.zeros(len(groups))
    g0 = 0
    for nl in nls:
        for j in range(nl - 1):
            g, h = g0 + j, g0 + j + 1
            d = p[h] - p[g]
            w = abs(lams[h] - lams[g]) / (0.5 * (lams[g] + lams[h]))
            sb = 0.5 * (s[g] + s[h])
            M += w * sb / abs(d)
            ds[g] += 0.5 * w / abs(d)
            ds[h] += 0.5 * w / abs(d)
            dp[h] += -w * sb / (abs(d) * d)
            dp[g] -= -w * sb / (abs(d) * d)
        g0 += nl
    rX, rY = np.zeros(X.size), np.zeros(X.size)
    for g, i in enumerate(groups):
        dq = dp[g] / i.size + ds[g] * (q[i] - p[g]) / (i.size * s[g])
        rX[i], rY[i] = u[0] * dq, u[1] * dq
    return M, rX, rY


@pytest.mark.parametrize("n_lambda", [64, 300])
def test_resolution_merit_and_seeds_against_numpy(n_lambda):
    """rtb_adjoint_resolution_merit on the same two beams, along a tilted
    dispersion direction: merit and seeds equal the numpy restatement; rays
    outside every beam get 0; a zero direction is refused."""
    adj, X, Y, good, groups, lams, outside, nls = _two_beam_forward(n_lambda)
    u = (0.8, -0.35)
    m_lib, gX, gY = adj.resolution_merit(lams, u)
    M, rX, rY = resolution_np(X, Y, [i[good[i]] for i in groups], lams, nls, u)
    assert abs(m_lib - M) <= 1e-11 * abs(M), (m_lib, M)
    _check_seeds(gX, gY, rX, rY, outside)
    with pytest.raises(RuntimeError):
        adj.resolution_merit(lams, (0.0, 0.0))
    adj.destroy()


def resolution_difference(Xp, Yp, Xm, Ym, groups, lams):
    """M(+) - M(-) of the resolution merit along x for two forwards on the same
    rays, from per-ray differences (Xp - Xm is exact for nearby doubles) so
    that it keeps its digits where M is far larger than the difference:
    per pair, s/|d| moves by (ds |d-| - s- d|d|) / (|d+| |d-|), with the width
    difference ds = (s+^2 - s-^2) / (s+ + s-) from the products of the
    per-ray differences and sums."""
    p, s, dp, ds = [], [], [], []
    for i in groups:
        xp, xm = Xp[i], Xm[i]
        dx = xp - xm
        pp, pm, dmean = xp.mean(), xm.mean(), dx.mean()
        up, um = xp - pp, xm - pm
        sp, sm = np.sqrt(np.mean(up * up)), np.sqrt(np.mean(um * um))
        dvar = np.mean((dx - dmean) * (up + um))  # s+^2 - s-^2
        p.append(pm)
        s.append(sm)
        dp.append(dmean)
        ds.append(dvar / (sp + sm))
    dM = 0.0
    for g in range(len(groups) - 1):
        h = g + 1
        w = abs(lams[h] - lams[g]) / (0.5 * (lams[g] + lams[h]))
        dm_, dd = p[h] - p[g], dp[h] - dp[g]
        dpl = dm_ + dd
        sbar_m, dsbar = 0.5 * (s[g] + s[h]), 0.5 * (ds[g] + ds[h])
        dM += w * (dsbar * abs(dm_) - sbar_m * np.sign(dm_) * dd) / (abs(dpl) * abs(dm_))
    return dM


def test_resolution_merit_gradient_matches_central_differences():
    """The gradient of the spectral-resolution merit by one forward, the
    merit's seeds and one backward against central differences of the FP64
    forward (relative step 1e-6) on C4 at 1e5 rays, both over the rays good at
    theta0 and at every difference point: within 1e-6 relative.  Where no ray
    changes its fate between those points, the library's own seeds
    (rtb_adjoint_resolution_merit) give the same gradient."""
    _, _, beams, n, rays, adj = setup(1600)
    theta0 = adj.theta()
    P = len(theta0)
    h = steps(theta0)
    lam = np.linspace(S.C4_LAMBDA[0], S.C4_LAMBDA[1], S.C4_NLAMBDA)
    groups = [np.arange(j, n, S.C4_NLAMBDA) for j in range(S.C4_NLAMBDA)]
    adj.forward(None, rays)
    good0 = adj.flag.cpu().numpy() == 1
    mask = good0.copy()
    pts = []
    for j in range(P):
        for sgn in (1.0, -1.0):
            t = theta0.copy()
            t[j] += sgn * h[j]
            st, _ = adj.forward(t, rays)
            assert st == ffi.OK
            mask &= adj.flag.cpu().numpy() == 1
            pts.append((adj.X.cpu().numpy(), adj.Y.cpu().numpy()))
    gm = [i[mask[i]] for i in groups]
    merit = lambda X, Y: resolution_np(X, Y, gm, lam, [S.C4_NLAMBDA], (1.0, 0.0))  # noqa: E731
    fd = np.array([resolution_difference(*pts[2 * j], *pts[2 * j + 1], gm, lam) / (2 * h[j]) for j in range(P)])
    del pts
    adj.forward(None, rays)
    M, rX, rY = merit(adj.X.cpu().numpy(), adj.Y.cpu().numpy())
    g = adj.backward(torch.as_tensor(rX, device="cuda"), torch.as_tensor(rY, device="cuda"))
    rel = np.abs(g - fd) / np.abs(fd)
    print("resolution merit", M, "rays changing fate", int((good0 & ~mask).sum()), "rel err", rel.max())
    assert np.all(np.abs(fd) > 0)
    assert rel.max() <= 1e-6, (int(np.argmax(rel)), rel.max())
    if np.array_equal(mask, good0):
        m_lib, gX, gY = adj.resolution_merit(lam)
        assert abs(m_lib - M) <= 1e-11 * abs(M)
        assert np.allclose(adj.backward(gX, gY), g, rtol=1e-9, atol=0)
    adj.destroy()
