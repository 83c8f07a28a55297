"""Parity of the CUDA engine with the CPU oracle (GPU tests).

The plain FP64 engine (drop-in calls, per-surface trace, fused trace) is
compiled with --fmad=false and must equal the oracle bit for bit (NaN
payloads aside) on the same inputs: positions, direction cosines,
wavelengths, lost flags, lost stages, counts.
"""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle as O
import refharness as H
from rt_b200 import engine as E
from rt_b200 import ffi, schemes as S

pytestmark = pytest.mark.gpu

SCHEMES = {
    "c0": (S.littrow_free, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c4": (S.littrow_free_asphere, dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.7)), ()),
    "c1": (S.echelle, dict(n_lambda=64, radius=25.0, lam_range=(0.38, 0.90)), (41, 1)),
    "mirrors": (lambda: S.coverage_schemes()["mirrors"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
    "lenses": (lambda: S.coverage_schemes()["lenses"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
    "gratings": (lambda: S.coverage_schemes()["gratings"], dict(n_lambda=5, radius=10.0, lam_range=(0.4, 0.8)), ()),
}
FIXES = [0, ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP, ffi.FIX_TORIC_SIGN | ffi.FIX_TORIC_STEP | ffi.FIX_ASPHERE_ROOT]


def same_bits(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    eq = a.view(np.uint64) == b.view(np.uint64)
    return bool(np.all(eq | (np.isnan(a) & np.isnan(b))))


def assert_rays_equal(dev_h, ora, fields=E.FIELDS):
    for f in fields:
        assert same_bits(getattr(dev_h, f), getattr(ora, f)), f
    assert np.array_equal(dev_h.flag, ora.flag)
    assert np.array_equal(dev_h.lost_stage, ora.lost_stage)


def _case(name, n_per=200, seed=99, n_beams=1):
    make, kw, orders = SCHEMES[name]
    beams = []
    first = 0
    for b in range(n_beams):
        bm = S.make_beam(first, n_per, kw["n_lambda"], kw["radius"], kw["lam_range"], seed + b, orders=orders)
        beams.append(bm)
        first += bm.n_rays
    return make(), beams, first


# ---------------------------------------------------------------------------
# beams

def test_generate_matches_oracle():
    beams = S.c1_beams(n_per_lambda=97)[:5]
    n = S.total_rays(beams)
    dev = E.generate(beams, n).to_host(O.HostRays)
    ora = O.generate(beams, n)
    assert_rays_equal(dev, ora)


def test_beam_random_and_lambda_dropin():
    L = E.lib()
    n = 5000
    X, Y, Z = (np.zeros(n) for _ in range(3))
    params = np.array([n, 1.0, 12.0])
    center = np.array([0.5, -0.25, 3.0])
    ffi.check(L.rtb_beam_random(0, ffi.dptr(params), ffi.dptr(center), C.c_size_t(n), ffi.dptr(X), ffi.dptr(Y),
                                ffi.dptr(Z), C.c_uint64(7), C.c_uint64(100)))
    oX, oY, oZ = (np.zeros(n) for _ in range(3))
    O.load().oracle_beam_random(0, ffi.dptr(params), ffi.dptr(center), C.c_size_t(n), ffi.dptr(oX), ffi.dptr(oY),
                                ffi.dptr(oZ), C.c_uint64(7), C.c_uint64(100))
    assert same_bits(X, oX) and same_bits(Y, oY) and same_bits(Z, oZ)
    r = np.hypot(X - 0.5, Y + 0.25)
    assert r.min() >= 1.0 and r.max() <= 12.0
    lam = np.zeros(64)
    rng = np.array([0.38, 0.9])
    ffi.check(L.rtb_uniform_range_beam(C.c_size_t(64), ffi.dptr(rng), ffi.dptr(lam)))
    olam = np.zeros(64)
    O.load().oracle_uniform_range_beam(C.c_size_t(64), ffi.dptr(rng), ffi.dptr(olam))
    assert same_bits(lam, olam)


# ---------------------------------------------------------------------------
# traces

@pytest.mark.parametrize("name", list(SCHEMES))
@pytest.mark.parametrize("engine", [ffi.ENGINE_PER_SURFACE, ffi.ENGINE_FUSED])
@pytest.mark.parametrize("fixes", FIXES)
def test_trace_matches_oracle(name, engine, fixes):
    specs, beams, n = _case(name, n_per=300, n_beams=3)
    cs_d = S.to_c(specs, E.spline_init)
    cs_o = S.to_c(specs, O.spline_init)
    ora = O.generate(beams, n)
    dev = E.DeviceRays.from_host(ora)
    st_o, stats_o, _ = O.trace(cs_o.surfaces, beams, ora, fixes=fixes)
    st_d, stats_d = E.trace(cs_d.surfaces, beams, dev, E.opts(engine=engine, fixes=fixes))
    assert st_d == st_o
    assert (stats_d.ray_surfaces, stats_d.n_good, stats_d.failed_beam, stats_d.failed_stage) == \
        (stats_o.ray_surfaces, stats_o.n_good, stats_o.failed_beam, stats_o.failed_stage)
    assert_rays_equal(dev.to_host(O.HostRays), ora)


def _cycle_rays():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "toric_cycles.npz"))
    st = z["state"]
    r = O.HostRays(st.shape[1])
    for f, row in zip(E.FIELDS[:6], st):
        getattr(r, f)[:] = row
    r.lambda_[:] = 0.5
    return r, z


@pytest.mark.parametrize("fixes", FIXES)
def test_toric_cycles_match_oracle(fixes):
    """Rays of the C1 fold whose toric iteration falls into a cycle and runs
    to the iteration cap: the CUDA engine skips whole periods of the cycle,
    the oracle runs every step; results must be the same bits."""
    rays, z = _cycle_rays()
    assert z["cycling_fixed"].sum() >= 1 and z["cycling_literal"].sum() >= 1
    p = np.zeros(16)
    p[:4] = z["params"][:4]
    out = []
    for fn in _pair("surface_intersection_fix"):
        r = rays.copy()
        nb = C.c_size_t(0)
        st = fn(ffi.TORIC, ffi.dptr(p), C.c_size_t(r.n), *(ffi.dptr(getattr(r, f)) for f in E.FIELDS[:6]),
                C.byref(nb), ffi.vptr(r.flag), C.c_uint(fixes))
        assert st == ffi.OK
        out.append((r, nb.value))
    (a, na), (b, nb_) = out
    assert na == nb_
    for f in ("X", "Y", "Z"):
        assert same_bits(getattr(a, f), getattr(b, f)), f
    assert np.array_equal(a.flag, b.flag)
    # the same rays through the trace engines, as a one-surface scheme
    specs = [S.SurfaceSpec(ffi.TORIC, ffi.MIRROR, params=tuple(z["params"][:4]), size=(1000.0, 0.0))]
    beams = [S.make_beam(0, rays.n, 1, 1.0, (0.5, 0.5), 1)]
    cs_o, cs_d = S.to_c(specs, O.spline_init), S.to_c(specs, E.spline_init)
    ora = rays.copy()
    st_o, stats_o, _ = O.trace(cs_o.surfaces, beams, ora, fixes=fixes)
    for engine in (ffi.ENGINE_PER_SURFACE, ffi.ENGINE_FUSED):
        dev = E.DeviceRays.from_host(rays)
        st_d, stats_d = E.trace(cs_d.surfaces, beams, dev, E.opts(engine=engine, fixes=fixes))
        assert st_d == st_o
        assert stats_d.ray_surfaces == stats_o.ray_surfaces
        assert_rays_equal(dev.to_host(O.HostRays), ora)


def test_fused_writes_only_xy_when_asked():
    specs, beams, n = _case("c0", n_per=500)
    cs = S.to_c(specs, E.spline_init)
    rays = E.generate(beams, n)
    full = rays.copy()
    E.trace(cs.surfaces, beams, full, E.opts())
    before = rays.copy()
    st, _ = E.trace(cs.surfaces, beams, rays, E.opts(state_out=0))
    assert st == ffi.OK
    a, b, c = rays.to_host(O.HostRays), full.to_host(O.HostRays), before.to_host(O.HostRays)
    assert same_bits(a.X, b.X) and same_bits(a.Y, b.Y)
    assert same_bits(a.cZ, c.cZ) and same_bits(a.Z, c.Z)


def test_trace_host_matches_device():
    specs, beams, n = _case("c1", n_per=400, n_beams=4)
    cs = S.to_c(specs, E.spline_init)
    dev = E.generate(beams, n)
    h = E.PinnedRays(n)
    src = dev.to_host(O.HostRays)
    for f in E.FIELDS:
        getattr(h, f)[:] = getattr(src, f)
    st_d, stats_d = E.trace(cs.surfaces, beams, dev, E.opts())
    st_h, stats_h = E.trace_host(cs.surfaces, beams, h, E.opts())
    assert st_d == st_h == ffi.OK
    assert stats_d.ray_surfaces == stats_h.ray_surfaces and stats_d.n_good == stats_h.n_good
    d = dev.to_host(O.HostRays)
    for f in ("X", "Y", "Z", "cX", "cY", "cZ"):
        assert same_bits(getattr(h, f), getattr(d, f)), f
    assert np.array_equal(h.flag, d.flag) and np.array_equal(h.lost_stage, d.lost_stage)
    h.free()


def test_out_of_range_wavelength_is_an_error():
    specs = S.coverage_schemes()["lenses"]
    beams = [S.make_beam(0, 10, 1, 5.0, (1.2, 1.2), 3)]  # glass table ends at 0.95 um
    cs = S.to_c(specs, E.spline_init)
    rays = E.generate(beams, 10)
    st, _ = E.trace(cs.surfaces, beams, rays, E.opts())
    assert st == ffi.OUT_OF_RANGE


def test_no_intersections_status():
    specs = [S.SurfaceSpec(ffi.PLANE, ffi.DETECTOR, distance=(0.0, 0.0, -10.0))]
    beams = [S.make_beam(0, 10, 1, 5.0, (0.5, 0.5), 1)]
    cs = S.to_c(specs, E.spline_init)
    for eng in (ffi.ENGINE_PER_SURFACE, ffi.ENGINE_FUSED):
        rays = E.generate(beams, 10)
        st, stats = E.trace(cs.surfaces, beams, rays, E.opts(engine=eng))
        assert st == ffi.NO_INTERSECTIONS and stats.failed_stage == 0


# ---------------------------------------------------------------------------
# order, frame

@pytest.mark.parametrize("name", ["c1", "mirrors", "gratings"])
def test_reference_order_matches_oracle(name):
    specs, beams, n = _case(name, n_per=150, n_beams=3)
    cs = S.to_c(specs, E.spline_init)
    rays = E.generate(beams, n)
    E.trace(cs.surfaces, beams, rays, E.opts())
    order = E.reference_order(beams, 3 * len(specs), rays).cpu().numpy().astype(np.int64)
    ls = rays.lost_stage.cpu().numpy()
    for b in beams:
        a, z = int(b.first_ray), int(b.first_ray + b.n_rays)
        o_ref, _ = O.reference_order(ls[a:z], 3 * len(specs))
        assert np.array_equal(order[a:z], o_ref.astype(np.int64))


def test_ccd_frame_counts_exact():
    specs, beams, n = _case("c0", n_per=4000)
    cs = S.to_c(specs, E.spline_init)
    rays = E.generate(beams, n)
    E.trace(cs.surfaces, beams, rays, E.opts())
    ccd = S.ccd(S.C0_CCD)
    counts, outside = E.ccd_frame(rays, ccd)
    h = rays.to_host(O.HostRays)
    ref_counts, ref_out = O.ccd_frame(h, ccd)
    assert np.array_equal(counts.cpu().numpy().view(np.uint32), ref_counts)
    assert int(outside.item()) == ref_out
    assert int(counts.sum().item()) + ref_out == int((h.flag == 1).sum())
    # fused epilogue gives the same frame
    import torch
    rays2 = E.generate(beams, n)
    c2 = torch.zeros_like(counts)
    o2 = torch.zeros_like(outside)
    st, _ = E.trace(cs.surfaces, beams, rays2, E.opts(ccd=ccd, counts=c2, n_outside=o2))
    assert st == ffi.OK
    assert torch.equal(c2, counts) and int(o2.item()) == ref_out


# ---------------------------------------------------------------------------
# drop-in calls

def _rays_for(name, n_per=200):
    specs, beams, n = _case(name, n_per=n_per)
    return specs, O.generate(beams, n)


def _pair(fn_name, *args_builder):
    return getattr(E.lib(), "rtb_" + fn_name), getattr(O.load(), "oracle_" + fn_name)


@pytest.mark.parametrize("params,cls", [
    ((0.0, 0.0, 0), ffi.PLANE), ((-1 / 800.0, -1.0, 0), ffi.CONIC), ((1 / 300.0, -0.4, 0), ffi.CONIC),
    ((-1 / 300.0, 0.3, 0), ffi.CONIC), ((1 / 150.0, 0.0, 5, 0.0, 1e-9, -2e-13, 1e-17, 0.0), ffi.CONIC),
    ((0.0, 0.0, 2, 1e-4, -3e-8), ffi.CONIC), ((-1 / 900.0, 0.2, 0, -1 / 800.0), ffi.TORIC),
])
def test_dropin_intersection(params, cls):
    rays = O.generate([S.make_beam(0, 3000, 1, 20.0, (0.5, 0.5), 5, field=(0.01, -0.02),
                                   center=(0.0, 0.0, -50.0))], 3000)
    p = np.zeros(16)
    p[:len(params)] = params
    out = []
    for fn in _pair("surface_intersection"):
        r = rays.copy()
        nb = C.c_size_t(0)
        st = fn(cls, ffi.dptr(p), C.c_size_t(r.n), *(ffi.dptr(getattr(r, f)) for f in E.FIELDS[:6]), C.byref(nb),
                ffi.vptr(r.flag))
        assert st == ffi.OK
        out.append((r, nb.value))
    (a, na), (b, nb_) = out
    assert na == nb_
    for f in ("X", "Y", "Z"):
        assert same_bits(getattr(a, f), getattr(b, f)), f
    assert np.array_equal(a.flag, b.flag)


@pytest.mark.parametrize("cls,params", [(ffi.PLANE, (0, 0, 0)), (ffi.CONIC, (-1 / 500.0, -0.5, 2, 1e-6, 1e-10)),
                                        (ffi.TORIC, (-1 / 900.0, 0.2, 1, 1e-7, -1 / 800.0))])
def test_dropin_reflection_refraction_diffraction(cls, params):
    specs, rays = _rays_for("c0", n_per=400)
    rays.X *= 0.5
    rays.Y *= 0.5
    rays.cX[:] = 0.05 * np.sin(np.arange(rays.n))
    rays.cY[:] = 0.04 * np.cos(np.arange(rays.n))
    rays.cZ[:] = np.sqrt(1 - rays.cX ** 2 - rays.cY ** 2)
    p = np.zeros(16)
    p[:len(params)] = params
    gx, gy = S.glass_table()
    t_d, t_o = ffi.TableHolder(gx, gy), ffi.TableHolder(gx, gy)
    t_d.y2[:] = E.spline_init(gx, gy)
    t_o.y2[:] = O.spline_init(gx, gy)
    one = ffi.TableHolder(value=1.0)
    res = []
    for fn in _pair("surface_reflection"):
        r = rays.copy()
        assert fn(cls, ffi.dptr(p), C.c_size_t(r.n), *(ffi.dptr(getattr(r, f)) for f in E.FIELDS[:6])) == ffi.OK
        res.append(r)
    assert all(same_bits(getattr(res[0], f), getattr(res[1], f)) for f in ("cX", "cY", "cZ"))
    for (fd, fo), tabs in [(_pair("surface_refraction"), ((one, t_d), (one, t_o))),
                           (_pair("surface_refraction"), ((t_d, one), (t_o, one)))]:
        res = []
        for fn, (n1, n2) in zip((fd, fo), tabs):
            r = rays.copy()
            nb = C.c_size_t(0)
            assert fn(cls, ffi.dptr(p), C.c_size_t(r.n), *(ffi.dptr(getattr(r, f)) for f in E.FIELDS[:6]),
                      ffi.dptr(r.lambda_), C.byref(n1.table), C.byref(n2.table), C.byref(nb),
                      ffi.vptr(r.flag)) == ffi.OK
            res.append((r, nb.value))
        assert res[0][1] == res[1][1]
        assert all(same_bits(getattr(res[0][0], f), getattr(res[1][0], f)) for f in ("cX", "cY", "cZ"))
        assert np.array_equal(res[0][0].flag, res[1][0].flag)
    for gtype, order, d in [(ffi.REFLECTIVE, 1, 1.6667), (ffi.REFLECTIVE, -3, 1.2), (ffi.TRANSPARENT, 1, 2.0),
                            (ffi.TRANSPARENT, 4, 3.0)]:
        res = []
        for fn, (n1, n2) in zip(_pair("surface_diffration"), ((one, t_d), (one, t_o))):
            r = rays.copy()
            nb = C.c_size_t(0)
            assert fn(cls, gtype, ffi.dptr(p), C.c_long(order), C.c_double(d), C.c_size_t(r.n),
                      *(ffi.dptr(getattr(r, f)) for f in E.FIELDS[:6]), ffi.dptr(r.lambda_), C.byref(n1.table),
                      C.byref(n2.table), C.byref(nb), ffi.vptr(r.flag)) == ffi.OK
            res.append((r, nb.value))
        assert res[0][1] == res[1][1]
        assert all(same_bits(getattr(res[0][0], f), getattr(res[1][0], f)) for f in ("cX", "cY", "cZ"))
        assert np.array_equal(res[0][0].flag, res[1][0].flag)


def test_dropin_transform_normalize_aperture_rearrange_ccd():
    specs, rays = _rays_for("c1", n_per=300)
    ang = np.array([0.3, -1.2, 2.5])
    dist = np.array([1.0, -2.0, 300.0])
    res = []
    for fn in _pair("beam_transform"):
        r = rays.copy()
        assert fn(C.c_size_t(r.n), ffi.dptr(ang), ffi.dptr(dist), *(ffi.dptr(getattr(r, f)) for f in E.FIELDS[:6])) == 0
        res.append(r)
    assert all(same_bits(getattr(res[0], f), getattr(res[1], f)) for f in E.FIELDS[:6])
    base = res[0]
    base.cX *= 3.0
    base.cY -= 0.1
    res = []
    for fn in _pair("normalize"):
        r = base.copy()
        assert fn(C.c_size_t(r.n), ffi.dptr(r.cX), ffi.dptr(r.cY), ffi.dptr(r.cZ)) == 0
        res.append(r)
    assert all(same_bits(getattr(res[0], f), getattr(res[1], f)) for f in ("cX", "cY", "cZ"))
    for shade in (0, 1):
        for shape, size in ((0, (15.0, 0.0)), (1, (20.0, 12.0))):
            res = []
            for fn in _pair("apply_constrains"):
                r = rays.copy()
                nb = C.c_size_t(0)
                sz, ce = np.array(size), np.array([1.0, -0.5])
                assert fn(shade, shape, ffi.dptr(sz), ffi.dptr(ce), C.c_size_t(r.n), ffi.dptr(r.X), ffi.dptr(r.Y),
                          ffi.vptr(r.flag), C.byref(nb)) == 0
                res.append((r, nb.value))
            assert res[0][1] == res[1][1] and np.array_equal(res[0][0].flag, res[1][0].flag)
            flagged = res[0][0]
    res = []
    for fn in _pair("rearrange"):
        r = flagged.copy()
        ng = C.c_size_t(r.n)
        assert fn(C.byref(ng), *(ffi.dptr(getattr(r, f)) for f in E.FIELDS), ffi.vptr(r.flag)) == 0
        res.append((r, ng.value))
    assert res[0][1] == res[1][1]
    assert all(same_bits(getattr(res[0][0], f), getattr(res[1][0], f)) for f in E.FIELDS)
    assert np.array_equal(res[0][0].flag, res[1][0].flag)
    xs = rays.X * 2
    ys = rays.Y * 2 - 3
    xs[:3] = (np.nan, -100.0, 1e12)
    out = []
    for fn in _pair("ccd_coordinates"):
        ix = np.zeros(rays.n, dtype=np.uint32)
        iy = np.zeros(rays.n, dtype=np.uint32)
        assert fn(C.c_size_t(rays.n), ffi.dptr(xs), ffi.dptr(ys), C.c_double(30.72), C.c_double(30.72),
                  C.c_double(0.015), C.c_double(0.015), ffi.vptr(ix), ffi.vptr(iy)) == 0
        out.append((ix, iy))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][0][0] == 0x80000000 and out[0][0][1] == 0 and out[0][0][2] == 0xFFFFFFFF


def test_dropin_ccd_image_and_qe():
    n = 20000
    rng = np.random.default_rng(3)
    lam = rng.uniform(0.36, 0.74, n)
    ix = rng.integers(0, 70, n).astype(np.uint32)
    iy = rng.integers(0, 70, n).astype(np.uint32)
    qx, qy = S.qe_table()
    q_d, q_o = ffi.TableHolder(qx, qy), ffi.TableHolder(qx, qy)
    q_d.y2[:] = E.spline_init(qx, qy)
    q_o.y2[:] = O.spline_init(qx, qy)
    spec = ffi.TableHolder(value=2.5)
    imgs = []
    for fn, q in zip(_pair("compute_ccd_image"), (q_d, q_o)):
        img = np.zeros(64 * 64)
        out = np.zeros(1, dtype=np.uint64)
        assert fn(C.c_size_t(n), ffi.vptr(ix), ffi.vptr(iy), ffi.dptr(lam), C.byref(q.table), C.byref(spec.table),
                  C.c_size_t(64), C.c_size_t(64), C.c_double(0.015), C.c_double(0.015), ffi.dptr(img),
                  ffi.vptr(out)) == 0
        imgs.append((img, int(out[0])))
    assert imgs[0][1] == imgs[1][1] > 0
    np.testing.assert_allclose(imgs[0][0], imgs[1][0], rtol=1e-13, atol=0)
    specs = []
    for fn, q in zip(_pair("surface_QE"), (q_d, q_o)):
        sp = np.linspace(1, 2, n)
        assert fn(C.c_size_t(n), ffi.dptr(lam), ffi.dptr(sp), C.byref(q.table)) == 0
        specs.append(sp)
    assert same_bits(specs[0], specs[1])


# ---------------------------------------------------------------------------
# the reference's host classes over the B200 engine (shim)

@pytest.mark.parametrize("name", ["c0", "c1", "mirrors", "lenses", "gratings"])
def test_shim_dropin_equals_reference_host_classes_on_oracle(name):
    """harness_b200 (reference Beam/Surface/TabulatedFunction + shim + this
    library) writes the same .dat as harness_cpu (same classes + oracle)."""
    if H.harness("b200") is None or H.harness("cpu") is None:
        pytest.skip("oracle/_ref harnesses not built")
    specs, beams, n = _case(name, n_per=60)
    rays = O.generate(beams, n)
    orders = list(beams[0].orders)[:beams[0].n_orders]
    rc_b, out_b = H.run_trace("b200", specs, orders, rays)
    rc_c, out_c = H.run_trace("cpu", specs, orders, rays)
    assert rc_b == rc_c
    if rc_b == 0:
        assert out_b[:3] == out_c[:3]
        assert same_bits(out_b[3], out_c[3])
