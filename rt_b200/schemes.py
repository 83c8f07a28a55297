"""Spectrograph schemes and synthetic beams of the benchmark configurations.

A scheme is a list of `SurfaceSpec`, the fields of one <surface> element of
the reference's scheme XML (common-lib/scheme.cpp:416-664); `to_c()` turns it
into the rtb_surface array of include/rtb.h.  The geometry the benchmark
configurations leave open (distances, tilts, apertures, the glass and QE
tables) is fixed here and seeded.

Configurations:
  * C0  `littrow_free()`: parabolic collimator R=-800 (k=-1) at z=400, plane
        600 l/mm grating order +1 tilted 10 deg about x, spherical camera
        R=-600, plane CCD 2048^2 x 15 um; 5 wavelengths 0.400..0.700 um.
  * C1  `echelle()`: off-axis parabola R=-1600 (k=-1), echelle 31.6 l/mm
        (orders 30..60, one range per order), cross-disperser 300 l/mm order 1
        turned 90 deg about z, toric fold Rx=-2000 Ry=-2100, even-asphere lens
        R=150/-400 with A4..A10 ~ N(0, 1e-7*10^-3k) and a 61-knot glass n(l),
        plane CCD 4096^2 x 15 um; 64 wavelengths 0.380..0.900 um.
  * C3  `c3_beams()`: 512 beams of log-uniform size (1e3..1e6 rays), each
        with its own wavelength, field angle and echelle order, through C1.
  * C4  `littrow_free_asphere()`: C0 extended with an even-asphere field
        flattener before the CCD; 64 wavelengths 0.400..0.700 um.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import ffi

SEED = 20141203  # master seed of every synthetic table and beam


# ---------------------------------------------------------------------------
# tables

def qe_table(seed: int = SEED) -> tuple[np.ndarray, np.ndarray]:
    """CCD QE: 41 knots over 0.35..0.75 um, values uniform in [0.6, 0.95]."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.35, 0.75, 41)
    return x, rng.uniform(0.6, 0.95, size=41)


def qe_table_wide(seed: int = SEED + 5) -> tuple[np.ndarray, np.ndarray]:
    """CCD QE for the echelle: 61 knots over 0.35..0.95 um, a broad hump
    0.9 - 1.2 (l - 0.6)^2 with a seeded ripple of +-0.02."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.35, 0.95, 61)
    return x, 0.9 - 1.2 * (x - 0.6) ** 2 + rng.uniform(-0.02, 0.02, size=61)


def glass_table() -> tuple[np.ndarray, np.ndarray]:
    """Camera-lens glass n(lambda): 61 knots over 0.35..0.95 um, a Cauchy law
    n = 1.5046 + 0.00420/l^2 (a borosilicate crown)."""
    x = np.linspace(0.35, 0.95, 61)
    return x, 1.5046 + 0.00420 / (x * x)


# ---------------------------------------------------------------------------
# surfaces

@dataclass
class SurfaceSpec:
    cls: int
    type: int
    shape: int = ffi.CIRCLE
    params: Sequence[float] = (0.0, 0.0, 0.0)
    size: Sequence[float] = (1000.0, 1000.0)
    center: Sequence[float] = (0.0, 0.0)
    distance: Sequence[float] = (0.0, 0.0, 0.0)
    angles: Sequence[float] = (0.0, 0.0, 0.0)      # degrees about y, x, z
    grating_type: int = ffi.REFLECTIVE
    order: int = 0
    gr_const: float = 0.0                          # microns
    n1: object = 1.0                               # float or (x, y) table
    n2: object = 1.0
    comment: str = ""
    # throughput (Scheme::ComputeQE): qe_curve as a float or (x, y) table,
    # None for none; grating blaze parameters in degrees, rule_params as
    # () for none, (v,) or (start, stop)
    qe: object = None
    alpha: float = 0.0
    gamma: float = 0.0
    blaze: float = 0.0
    rule_params: Sequence[float] = ()


def frame_towards(p: Sequence[float], v: Sequence[float]) -> tuple[list, list]:
    """Distance and angles (deg) of a surface frame whose origin is p and whose
    +z axis is the unit direction v, both given in the current frame, for the
    reference's transform (translation, then rotations about y, x, z,
    cuda_engine/rt_cuda_engine_beam.cu:416-579)."""
    vx, vy, vz = v
    rho = math.hypot(vx, vz)
    ay = math.degrees(math.atan2(vx, vz))
    ax = math.degrees(math.atan2(vy, rho))
    return [float(p[0]), float(p[1]), float(p[2])], [ay, ax, 0.0]


SplineFn = Callable[[np.ndarray, np.ndarray], np.ndarray]


class CScheme:
    """rtb_surface array built from specs; owns the table arrays."""

    def __init__(self, specs: Sequence[SurfaceSpec], spline: SplineFn):
        self.specs = list(specs)
        self.holders = []
        self.array = (ffi.Surface * len(self.specs))()
        for k, s in enumerate(self.specs):
            c = self.array[k]
            c.cls, c.type, c.shape, c.grating_type = s.cls, s.type, s.shape, s.grating_type
            c.order, c.gr_const = int(s.order), float(s.gr_const)
            if len(s.params) > ffi.MAX_PARAMS:
                raise ValueError("too many surface parameters")
            for i, v in enumerate(s.params):
                c.params[i] = float(v)
            c.size[0], c.size[1] = (float(s.size[0]), float(s.size[1] if len(s.size) > 1 else 0.0))
            c.center[0], c.center[1] = float(s.center[0]), float(s.center[1])
            for i in range(3):
                c.distance[i] = float(s.distance[i])
                c.angles_deg[i] = float(s.angles[i])
            c.n1 = self._table(s.n1, spline)
            c.n2 = self._table(s.n2, spline)

    def _table(self, t, spline: SplineFn) -> ffi.Table:
        if isinstance(t, (int, float)):
            h = ffi.TableHolder(value=float(t))
        else:
            h = ffi.TableHolder(x=t[0], y=t[1])
            h.y2[:] = spline(h.x, h.y)
        self.holders.append(h)
        return h.table

    def __len__(self) -> int:
        return len(self.specs)

    @property
    def surfaces(self):
        """The rtb_surface structs; each keeps this scheme (and so the table
        arrays its pointers refer to) alive."""
        out = list(self.array)
        for s in out:
            s._owner = self
        return out

    def n_gratings(self) -> int:
        return sum(1 for s in self.specs if s.type == ffi.GRATING)

    def non_aux(self) -> int:
        return sum(1 for s in self.specs if s.type != ffi.AUX_TYPE)


def to_c(specs: Sequence[SurfaceSpec], spline: SplineFn) -> CScheme:
    return CScheme(specs, spline)


QE_TYPES = (ffi.MIRROR, ffi.LENS, ffi.GRATING, ffi.DETECTOR)


class CQe:
    """rtb_qe_surface array of the surfaces Scheme::ComputeQE takes
    (scheme.cpp:1140-1209: non-AUX MIRROR, LENS, GRATING and DETECTOR
    surfaces, each with a qe_curve); owns the table arrays."""

    def __init__(self, specs: Sequence[SurfaceSpec], spline: SplineFn):
        self.specs = [s for s in specs if s.cls != ffi.AUX_CLASS and s.type in QE_TYPES]
        self.holders = []
        self.array = (ffi.QeSurface * max(1, len(self.specs)))()
        for k, s in enumerate(self.specs):
            if s.qe is None:
                raise ValueError(f"surface {k} has no qe_curve")
            c = self.array[k]
            c.type = s.type
            c.qe = CScheme._table(self, s.qe, spline)
            if s.type == ffi.GRATING:
                c.order, c.gr_const = int(s.order), float(s.gr_const)
                c.alpha_deg, c.gamma_deg, c.blaze_deg = float(s.alpha), float(s.gamma), float(s.blaze)
                rp = list(s.rule_params)
                rp = [0.0, 1.0] if not rp else ([0.0, rp[0]] if len(rp) == 1 else rp[:2])
                c.rule_start, c.rule_stop = float(rp[0]), float(rp[1])

    def __len__(self) -> int:
        return len(self.specs)


def qe_surfaces(specs: Sequence[SurfaceSpec], spline: SplineFn) -> CQe:
    return CQe(specs, spline)


# ---------------------------------------------------------------------------
# beams

def make_beam(first_ray: int, n_per_lambda: int, n_lambda: int, radius: float, lam_range,
              seed: int, orders: Sequence[int] = (), field=(0.0, 0.0), center=(0.0, 0.0, 0.0)) -> ffi.Beam:
    b = ffi.Beam()
    b.first_ray = first_ray
    b.n_rays = n_per_lambda * n_lambda
    b.n_orders = len(orders)
    for i, o in enumerate(orders):
        b.orders[i] = int(o)
    b.shape = ffi.CIRCLE
    b.disk[0], b.disk[1], b.disk[2] = float(n_per_lambda), 0.0, float(radius)
    for i in range(3):
        b.center[i] = float(center[i])
    b.range[0], b.range[1] = float(lam_range[0]), float(lam_range[1])
    b.n_lambda = n_lambda
    b.field[0], b.field[1] = float(field[0]), float(field[1])
    b.seed = seed
    return b


# ---------------------------------------------------------------------------
# C0: Littrow-free single-beam spectrograph

C0_LAMBDA = (0.400, 0.700)
C0_NLAMBDA = 5
C0_RADIUS = 10.0
C0_CCD = dict(xsize=30.72, ysize=30.72, xdim=2048, ydim=2048, xpix=0.015, ypix=0.015)


def littrow_free() -> list[SurfaceSpec]:
    """C0 scheme.  The beam (disk r=10 mm at z=0, along +z) meets the
    parabola (R=-800, k=-1) at z=400, converges through its focus 400 mm
    back, meets the grating 700 mm after the parabola (tilted 10 deg about x),
    the camera mirror 600 mm further on and the CCD in the camera's image of
    the focus.  Distances along the chief ray of 0.55 um."""
    par = SurfaceSpec(ffi.CONIC, ffi.MIRROR, params=(-1 / 800.0, -1.0, 0), size=(40.0, 0.0),
                      distance=(0.0, 0.0, 400.0), comment="collimator", qe=0.92)
    gr = SurfaceSpec(ffi.PLANE, ffi.GRATING, shape=ffi.RECTANGLE, size=(80.0, 80.0),
                     distance=(0.0, 0.0, -700.0), angles=(180.0, 10.0, 0.0), order=1,
                     gr_const=1.0 / 0.6, comment="grating 600 l/mm", qe=0.9, alpha=10.0, gamma=0.0, blaze=9.5)
    cam_d, cam_a = C0_FRAMES["camera"]
    cam = SurfaceSpec(ffi.CONIC, ffi.MIRROR, params=(-1 / 600.0, 0.0, 0), size=(80.0, 0.0),
                      distance=cam_d, angles=cam_a, comment="camera", qe=0.92)
    ccd_d, ccd_a = C0_FRAMES["ccd"]
    ccd = SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(30.72, 30.72),
                      distance=ccd_d, angles=ccd_a, comment="CCD 2048x2048 15um", qe=qe_table())
    return [par, gr, cam, ccd]


def c0_asphere_camera() -> list[SurfaceSpec]:
    """C0 with the camera mirror made an even asphere (A4, A6, A8 of small
    seeded values): a four-surface scheme with an iterative-asphere mirror."""
    s = littrow_free()
    rng = np.random.default_rng(SEED + 4)
    a = [0.0, float(rng.normal(0, 1e-10)), float(rng.normal(0, 1e-13)), float(rng.normal(0, 1e-16))]
    s[2].params = (-1 / 600.0, 0.0, len(a), *a)
    s[2].comment = "camera (even asphere)"
    return s


# C4's added surface: an even-asphere field flattener 15 mm in front of C0's
# CCD plane (same orientation), the CCD immersed in its glass and moved back
# to the paraxial refocus 15 mm x n(0.55 um).
C4_FLATTENER = dict(c=1 / 200.0, k=-0.5, A=(1e-6, -1e-9, 1e-12, -1e-15), back=15.0)
# C4 merit: centroid x target linear in lambda, x_t = X0 + X1 (lambda - 0.55)
C4_TARGET = (-0.3, -92.0)
C4_LAMBDA = (0.400, 0.700)
C4_NLAMBDA = 64


def _rot_matrix(ang_deg: Sequence[float]) -> np.ndarray:
    """R of the reference's transform (v_local = R v): rotations about y, x,
    z of the pairs (X,Z), (Y,Z), (X,Y) (rt_cuda_engine_beam.cu:320-350)."""
    K = 3.14159265359 / 180.0
    R = np.eye(3)
    for (i, j), a in zip(((0, 2), (1, 2), (0, 1)), ang_deg):
        c, s_ = math.cos(a * K), math.sin(a * K)
        M = np.eye(3)
        M[i, i], M[i, j], M[j, i], M[j, j] = c, -s_, s_, c
        R = M @ R
    return R


def littrow_free_asphere() -> list[SurfaceSpec]:
    """C4 scheme: C0 extended with one even-asphere surface, a field
    flattener (c=1/200, k=-0.5, A4..A10 = 1e-6, -1e-9, 1e-12, -1e-15) that
    takes the converging beam into glass 15 mm before C0's CCD plane; the CCD
    sits in the glass at the paraxial refocus."""
    s = littrow_free()
    ccd = s[3]
    f = C4_FLATTENER
    u = _rot_matrix(ccd.angles).T @ np.array([0.0, 0.0, 1.0])  # CCD axis in the camera frame
    gx, gy = glass_table()
    n55 = float(np.interp(0.55, gx, gy))
    d = [round(float(v), 9) for v in (np.array(ccd.distance) - f["back"] * u)]
    flat = SurfaceSpec(ffi.CONIC, ffi.LENS, params=(f["c"], f["k"], 5, 0.0, *f["A"]), size=(30.0, 0.0),
                       distance=d, angles=list(ccd.angles), n1=1.0, n2=(gx, gy),
                       comment="field flattener (even asphere)", qe=0.98)
    new_ccd = SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(30.72, 30.72),
                          distance=(0.0, 0.0, round(f["back"] * n55, 6)), comment="CCD 2048x2048 15um (in glass)",
                          qe=qe_table())
    return s[:3] + [flat, new_ccd]


def c4_beams(n_per_lambda: int = 156250, seed: int = SEED + 40) -> list[ffi.Beam]:
    """C4 beam: 64 wavelengths over 0.40-0.70 um, n_per_lambda rays each
    (1e7 rays by default), disk r=10 mm."""
    return [make_beam(0, n_per_lambda, C4_NLAMBDA, C0_RADIUS, C4_LAMBDA, seed)]


def c4_target_x(lam):
    return C4_TARGET[0] + C4_TARGET[1] * (np.asarray(lam) - 0.55)


def c4_params() -> list[tuple[int, int, int]]:
    """C4's 24 differentiable parameters as (surface, kind, index):
    curvatures (collimator, camera, flattener), conic constants (camera,
    flattener; the collimator's k = -1 selects the paraboloid algorithm and is
    held), the flattener's A4..A10, the grating's groove density, the
    collimator's decenter in y (its axial spacing does not act on a collimated
    beam), the axial spacings of the other four surfaces, and tilts about x
    and y of the grating, camera, flattener and CCD plus the collimator's tilt
    about x."""
    P = ffi
    p = [(0, P.PARAM_CURVATURE, 0), (2, P.PARAM_CURVATURE, 0), (3, P.PARAM_CURVATURE, 0),
         (2, P.PARAM_CONIC, 0), (3, P.PARAM_CONIC, 0)]
    p += [(3, P.PARAM_POLY, i) for i in (1, 2, 3, 4)]          # A4, A6, A8, A10 (a2..a5)
    p += [(1, P.PARAM_GROOVE_DENSITY, 0)]
    p += [(0, P.PARAM_DISTANCE, 1)]                            # collimator decenter in y
    p += [(k, P.PARAM_DISTANCE, 2) for k in range(1, 5)]       # axial spacings
    p += [(k, P.PARAM_ANGLE, i) for k in (1, 2, 3, 4) for i in (1, 0)]
    p += [(0, P.PARAM_ANGLE, 1)]
    assert len(p) == 24
    return p


def c0_beams(n_per_lambda: int = 20000, seed: int = SEED, first_ray: int = 0) -> list[ffi.Beam]:
    return [make_beam(first_ray, n_per_lambda, C0_NLAMBDA, C0_RADIUS, C0_LAMBDA, seed)]


# Frames of C0's camera and CCD (distance, angles) in the frame of the
# previous surface, found by tracing the chief ray (see design_frames()).
C0_FRAMES = {
    "camera": ([-198.0, -104.188907, -556.723155], [-160.421942, -4.0, 0.0]),
    "ccd": ([0.0, -47.560451, -452.507462], [180.0, -6.0, 0.0]),
}

# ---------------------------------------------------------------------------
# C1: cross-dispersed echelle

C1_LAMBDA = (0.380, 0.900)
C1_NLAMBDA = 64
C1_RADIUS = 25.0
C1_ORDERS = tuple(range(30, 61))
C1_CCD = dict(xsize=61.44, ysize=61.44, xdim=4096, ydim=4096, xpix=0.015, ypix=0.015)
# Frames (distance, angles) of C1's surfaces, each in the frame of the previous
# one, aimed along the chief ray of order 45 at 0.6284 um.
C1_FRAMES: dict = {
    "oap": ([0.0, -80.0, 1000.0], [0.0, 0.0, 0.0]),
    "echelle": ([0.0, 65.037406, -151.25187], [116.385776, -2.550993, 5.126721]),
    "xdisp": ([0.202434, 0.0, -149.999863], [179.922676, 0.0, 90.0]),
    "fold": ([-28.278, 0.0, -147.310403], [-169.133574, 12.0, 0.0]),
    "lens1": ([0.0, -31.186754, -146.72214], [180.0, -12.0, 0.0]),
    "lens2": ([0.0, 0.0, 12.0], [0.0, 0.0, 0.0]),
    "ccd": ([0.0, 0.0, 145.0], [0.0, 0.0, 0.0]),
}


def lens_asphere_coeffs(seed: int = SEED + 1) -> list[float]:
    """A4..A10 ~ N(0, 1e-7 * 10^-3k), k = 1..4, as polynomial terms a2..a5
    (a1, the r^2 term, is 0)."""
    rng = np.random.default_rng(seed)
    return [float(rng.normal(0.0, 1e-7 * 10.0 ** (-3 * k))) for k in range(1, 5)]


def echelle(glass=None) -> list[SurfaceSpec]:
    g = glass_table() if glass is None else glass
    a1 = lens_asphere_coeffs(SEED + 1)
    a2 = lens_asphere_coeffs(SEED + 2)
    f = C1_FRAMES
    return [
        SurfaceSpec(ffi.CONIC, ffi.MIRROR, params=(-1 / 1600.0, -1.0, 0), size=(140.0, 0.0),
                    distance=f["oap"][0], angles=f["oap"][1], comment="off-axis parabola", qe=0.92),
        SurfaceSpec(ffi.PLANE, ffi.GRATING, shape=ffi.RECTANGLE, size=(260.0, 120.0),
                    distance=f["echelle"][0], angles=f["echelle"][1], order=45, gr_const=1000.0 / 31.6,
                    comment="echelle 31.6 l/mm, blaze 63.5 deg", qe=0.85, alpha=64.5, gamma=4.0, blaze=63.5),
        SurfaceSpec(ffi.PLANE, ffi.GRATING, shape=ffi.RECTANGLE, size=(160.0, 160.0),
                    distance=f["xdisp"][0], angles=f["xdisp"][1], order=1, gr_const=1000.0 / 300.0,
                    comment="cross-disperser 300 l/mm", qe=0.9, alpha=10.0, gamma=0.0, blaze=4.3),
        SurfaceSpec(ffi.TORIC, ffi.MIRROR, params=(-1 / 2100.0, 0.0, 0, -1 / 2000.0), size=(110.0, 0.0),
                    distance=f["fold"][0], angles=f["fold"][1], comment="toric fold", qe=0.92),
        SurfaceSpec(ffi.CONIC, ffi.LENS, params=(1 / 150.0, 0.0, 5, 0.0, *a1), size=(75.0, 0.0),
                    distance=f["lens1"][0], angles=f["lens1"][1], n1=1.0, n2=g, comment="camera lens front",
                    qe=0.98),
        SurfaceSpec(ffi.CONIC, ffi.LENS, params=(-1 / 400.0, 0.0, 5, 0.0, *a2), size=(75.0, 0.0),
                    distance=f["lens2"][0], angles=f["lens2"][1], n1=g, n2=1.0, comment="camera lens back",
                    qe=0.98),
        SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(61.44, 61.44),
                    distance=f["ccd"][0], angles=f["ccd"][1], comment="CCD 4096x4096 15um", qe=qe_table_wide()),
    ]


def c1_rays_per_lambda(total: int = 100_000_000) -> int:
    """Rays per wavelength per order range: ceil(total / 31 / 64)."""
    return -(-total // (len(C1_ORDERS) * C1_NLAMBDA))


def c1_beams(n_per_lambda: int | None = None, seed: int = SEED, orders=C1_ORDERS) -> list[ffi.Beam]:
    """One beam per echelle order (range rows "0.38 0.90 m 1")."""
    n = c1_rays_per_lambda() if n_per_lambda is None else n_per_lambda
    beams, first = [], 0
    for i, m in enumerate(orders):
        beams.append(make_beam(first, n, C1_NLAMBDA, C1_RADIUS, C1_LAMBDA, seed + 1000 + i, orders=(m, 1)))
        first += n * C1_NLAMBDA
    return beams


def philox4x32_10(ctr: Sequence[int], key: int) -> tuple[int, int, int, int]:
    """Philox4x32-10 (Salmon et al., SC'11) on the host: the generator the
    device uses for ray positions, here for the per-beam draws of C3."""
    M0, M1, W0, W1, m = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85, 0xFFFFFFFF
    c0, c1, c2, c3 = (int(v) & m for v in ctr)
    k0, k1 = key & m, (key >> 32) & m
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & m, p1 & m, ((p0 >> 32) ^ c3 ^ k1) & m, p0 & m
        k0, k1 = (k0 + W0) & m, (k1 + W1) & m
    return c0, c1, c2, c3


def _u01(hi: int, lo: int) -> float:
    return float((((hi << 32) | lo) >> 11) + 1) * 2.0 ** -53


C3_BEAMS = 512
C3_COUNTS = (1e3, 1e6)          # log-uniform ray count per beam
C3_FIELD_DEG = 0.5              # field angle uniform in [-0.5, 0.5] deg in x and in y


def c3_beams(n_beams: int = C3_BEAMS, seed: int = SEED + 3, counts=C3_COUNTS, scale: float = 1.0) -> list[ffi.Beam]:
    """C3: independent beams through the C1 scheme, each with its own ray
    count (log-uniform in `counts`, times `scale`), wavelength (uniform over
    0.38-0.90 um), field angle (uniform +-0.5 deg in x and y, direction
    (tan fx, tan fy, 1) normalised) and echelle order (uniform 30..60).  The
    draws of beam b come from Philox4x32-10 with counters (b, 0..2, 0, 0) and
    key `seed`; the rays of beam b use seed + 1 + b."""
    beams, first = [], 0
    lo, hi = math.log(counts[0]), math.log(counts[1])
    for b in range(n_beams):
        r = philox4x32_10((b, 0, 0, 0), seed)
        s = philox4x32_10((b, 1, 0, 0), seed)
        n = max(1, int(round(math.exp(lo + (hi - lo) * _u01(r[0], r[1])) * scale)))
        lam = C1_LAMBDA[0] + (C1_LAMBDA[1] - C1_LAMBDA[0]) * _u01(r[2], r[3])
        fx = math.radians(C3_FIELD_DEG * (2.0 * _u01(s[0], s[1]) - 1.0))
        fy = math.radians(C3_FIELD_DEG * (2.0 * _u01(s[2], s[3]) - 1.0))
        t = philox4x32_10((b, 2, 0, 0), seed)
        m = C1_ORDERS[0] + min(len(C1_ORDERS) - 1, int(_u01(t[0], t[1]) * len(C1_ORDERS)))
        beams.append(make_beam(first, n, 1, C1_RADIUS, (lam, lam), seed + 1 + b, orders=(m, 1), field=(fx, fy)))
        first += n
    return beams


def total_rays(beams: Sequence[ffi.Beam]) -> int:
    return int(max(b.first_ray + b.n_rays for b in beams))


def ccd(cfg: dict) -> ffi.CCD:
    return ffi.CCD(cfg["xsize"], cfg["ysize"], cfg["xdim"], cfg["ydim"], cfg["xpix"], cfg["ypix"])


# ---------------------------------------------------------------------------
# Coverage schemes: small schemes that between them reach every surface
# class, type, aperture shape, intersection kind and action of the engine,
# with losses at every kind of stage.  Used by the parity tests.

def _glass_n():
    x, y = glass_table()
    return (x, y)


def coverage_schemes() -> dict[str, list[SurfaceSpec]]:
    g = _glass_n()
    mirrors = [
        SurfaceSpec(ffi.CONIC, ffi.MIRROR, params=(-1 / 500.0, 0.0, 0), size=(9.0, 0.0),
                    distance=(0.0, 0.0, 100.0), comment="spherical mirror, clips the beam edge"),
        SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE, distance=(0.0, 0.0, -60.0), angles=(180.0, 0.0, 0.0)),
        SurfaceSpec(ffi.TORIC, ffi.MIRROR, params=(-1 / 900.0, 0.2, 0, -1 / 800.0), size=(30.0, 0.0),
                    distance=(0.0, 0.0, 40.0), angles=(3.0, -2.0, 0.0), comment="toric mirror"),
        SurfaceSpec(ffi.PLANE, ffi.MIRROR, shape=ffi.RECTANGLE, size=(40.0, 40.0),
                    distance=(0.0, 0.0, -80.0), angles=(160.0, 5.0, 0.0), comment="plane fold"),
        SurfaceSpec(ffi.PLANE, ffi.STOP, shape=ffi.RECTANGLE, size=(16.0, 14.0), center=(3.47, -0.3),
                    distance=(11.714761, -1.364972, -27.584438), angles=(156.989684, -2.607805, 10.0),
                    comment="rectangular stop"),
        SurfaceSpec(ffi.PLANE, ffi.SHADE, size=(0.5, 0.0), center=(-4.6, 2.3),
                    distance=(0.0, 0.0, 20.0), comment="central obscuration"),
        SurfaceSpec(ffi.PLANE, ffi.SHADE, shape=ffi.RECTANGLE, size=(0.4, 30.0), center=(-4.0, 0.0),
                    distance=(0.0, 0.0, 5.0), comment="spider vane"),
        SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(30.72, 30.72),
                    distance=(0.0, 0.0, 60.0), comment="detector"),
    ]
    lenses = [
        SurfaceSpec(ffi.CONIC, ffi.LENS, params=(1 / 100.0, -0.5, 0), size=(12.0, 0.0),
                    distance=(0.0, 0.0, 50.0), n1=1.0, n2=1.5, comment="conic front, scalar indices"),
        SurfaceSpec(ffi.CONIC, ffi.LENS, params=(-1 / 200.0, 0.0, 3, 0.0, 2e-7, -1e-10), size=(12.0, 0.0),
                    distance=(0.0, 0.0, 8.0), n1=1.5, n2=g, comment="asphere, tabulated glass after"),
        SurfaceSpec(ffi.CONIC, ffi.LENS, params=(0.0, 0.0, 2, 1e-4, -3e-8), size=(12.0, 0.0),
                    distance=(0.0, 0.0, 6.0), n1=g, n2=1.0, comment="polynomial-only surface"),
        SurfaceSpec(ffi.PLANE, ffi.LENS, size=(30.0, 0.0), distance=(0.0, 0.0, 20.0), n1=1.0, n2=g,
                    comment="plane window front"),
        SurfaceSpec(ffi.PLANE, ffi.LENS, size=(30.0, 0.0), distance=(0.0, 0.0, 5.0), angles=(0.0, 41.0, 0.0),
                    n1=g, n2=1.0, comment="tilted window back (total internal reflection for part)"),
        SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(60.0, 60.0),
                    distance=(0.0, -34.79, 19.74), angles=(0.0, -60.4, 0.0), comment="detector"),
    ]
    gratings = [
        SurfaceSpec(ffi.PLANE, ffi.GRATING, size=(30.0, 0.0), distance=(0.0, 0.0, 30.0),
                    grating_type=ffi.TRANSPARENT, order=1, gr_const=2.0, n1=1.0, n2=g,
                    comment="transmission grating into glass"),
        SurfaceSpec(ffi.PLANE, ffi.LENS, size=(30.0, 0.0), distance=(0.0, 0.0, 5.0), n1=g, n2=1.0,
                    comment="glass back"),
        SurfaceSpec(ffi.CONIC, ffi.GRATING, params=(-1 / 400.0, 0.0, 0), size=(40.0, 0.0),
                    distance=(0.0, 0.0, 50.0), angles=(8.0, 0.0, 0.0), order=-1, gr_const=3.0,
                    comment="concave reflective grating"),
        SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE, distance=(0.0, 0.0, -40.0), angles=(180.0, 0.0, 0.0)),
        SurfaceSpec(ffi.CONIC, ffi.GRATING, params=(1 / 300.0, 0.0, 0), size=(40.0, 0.0),
                    distance=(0.0, 0.0, 0.0), grating_type=ffi.TRANSPARENT, order=1, gr_const=4.0,
                    n1=1.0, n2=1.0, comment="convex transmission grating"),
        SurfaceSpec(ffi.TORIC, ffi.GRATING, params=(-1 / 600.0, 0.0, 0, -1 / 500.0), size=(50.0, 0.0),
                    distance=(0.0, 0.0, 40.0), angles=(2.0, 0.0, 0.0), order=1, gr_const=5.0,
                    comment="toric reflective grating"),
        SurfaceSpec(ffi.AUX_CLASS, ffi.AUX_TYPE, distance=(0.0, 0.0, -30.0), angles=(180.0, 0.0, 0.0)),
        SurfaceSpec(ffi.TORIC, ffi.GRATING, params=(1 / 700.0, 0.0, 0, 1 / 650.0), size=(60.0, 0.0),
                    distance=(0.0, 0.0, 0.0), grating_type=ffi.TRANSPARENT, order=1, gr_const=6.0,
                    n1=1.0, n2=1.0, comment="toric transmission grating"),
        SurfaceSpec(ffi.PLANE, ffi.GRATING, size=(80.0, 0.0), distance=(0.0, 0.0, 30.0), order=2,
                    gr_const=1.3, comment="plane reflective grating, order 2 evanescent for red"),
        SurfaceSpec(ffi.PLANE, ffi.DETECTOR, shape=ffi.RECTANGLE, size=(80.0, 80.0),
                    distance=(-20.850663, 0.0, -21.569651), angles=(-135.971022, 0.0, 0.0), comment="detector"),
    ]
    return {"mirrors": mirrors, "lenses": lenses, "gratings": gratings}


# ---------------------------------------------------------------------------
# scheme files in the reference's format (common-lib/scheme.cpp:272-857)

_CLASS = {ffi.PLANE: "PLANE", ffi.CONIC: "CONIC", ffi.TORIC: "TORIC", ffi.AUX_CLASS: "AUX"}
_TYPE = {ffi.MIRROR: "MIRROR", ffi.LENS: "LENS", ffi.GRATING: "GRATING", ffi.STOP: "STOP", ffi.SHADE: "SHADE",
         ffi.DETECTOR: "DETECTOR", ffi.AUX_TYPE: "AUX"}


def _num(v) -> str:
    return " ".join(repr(float(x)) for x in (v if isinstance(v, (list, tuple, np.ndarray)) else [v]))


def write_table(path: str, x, y) -> None:
    """Two-column table file (TabulatedFunction::Load), newline-terminated."""
    with open(path, "w") as f:
        f.write("# lambda(um) value\n")
        for a, b in zip(x, y):
            f.write(f"{float(a)!r} {float(b)!r}\n")


def write_xml(path: str, specs: Sequence[SurfaceSpec], name: str, result_file: str, n_per_lambda: int,
              radius: float, ranges: Sequence[Sequence[float]], n_lambda: int = 0) -> None:
    """Write a scheme file the reference's ray-tracing program reads: values
    as element texts on one line, tables and (for more than one range) the
    range rows "w1 w2 order_1 .. order_G" in files beside it."""
    import os
    d = os.path.dirname(os.path.abspath(path))
    base = os.path.splitext(os.path.basename(path))[0]
    tables = {}

    def table_ref(t):
        if isinstance(t, (int, float)):
            return _num(t)
        key = (tuple(np.asarray(t[0]).tolist()), tuple(np.asarray(t[1]).tolist()))
        if key not in tables:
            fn = f"{base}_table{len(tables)}.txt"
            write_table(os.path.join(d, fn), t[0], t[1])
            tables[key] = fn
        return tables[key]

    L = ['<?xml version="1.0"?>', "<scheme>", "  <general>", f"    <name>{name}</name>",
         f"    <result_file>{result_file}</result_file>", "  </general>"]
    for s in specs:
        L.append("  <surface>")
        L.append(f"    <class>{_CLASS[s.cls]}</class>")
        if s.cls != ffi.AUX_CLASS:
            L.append(f"    <type>{_TYPE[s.type]}</type>")
            L.append(f"    <shape>{'CIRC' if s.shape == ffi.CIRCLE else 'RECT'}</shape>")
            L.append(f"    <params>{_num(list(s.params))}</params>")
            L.append(f"    <size>{_num(list(s.size) if s.shape == ffi.RECTANGLE else [s.size[0]])}</size>")
            L.append(f"    <center>{_num(list(s.center))}</center>")
        L.append(f"    <distance>{_num(list(s.distance))}</distance>")
        L.append(f"    <angles>{_num(list(s.angles))}</angles>")
        if s.comment:
            L.append(f"    <comment>{s.comment}</comment>")
        if s.type == ffi.GRATING:
            L.append(f"    <grating_type>{'TRANSPARENT' if s.grating_type == ffi.TRANSPARENT else 'REFLECTIVE'}"
                     "</grating_type>")
            L.append(f"    <order>{int(s.order)}</order>")
            L.append(f"    <const>{_num(s.gr_const)}</const>")
        if s.type in (ffi.GRATING, ffi.LENS):
            L.append(f"    <n1>{table_ref(s.n1)}</n1>")
            L.append(f"    <n2>{table_ref(s.n2)}</n2>")
        if s.qe is not None:
            L.append(f"    <qe_curve>{table_ref(s.qe)}</qe_curve>")
            if s.type == ffi.GRATING:
                L.append(f"    <alpha>{_num(s.alpha)}</alpha>")
                L.append(f"    <gamma>{_num(s.gamma)}</gamma>")
                L.append(f"    <blaze_angle>{_num(s.blaze)}</blaze_angle>")
                if len(s.rule_params):
                    L.append(f"    <rule_params>{_num(list(s.rule_params))}</rule_params>")
        L.append("  </surface>")
    if len(ranges) == 1 and len(ranges[0]) == 2:
        rng = _num(list(ranges[0]))
    else:
        rng = f"{base}_ranges.txt"
        with open(os.path.join(d, rng), "w") as f:
            f.write("# w1 w2 orders of the gratings in scheme order\n")
            for r in ranges:
                f.write(" ".join([repr(float(r[0])), repr(float(r[1]))] + [str(int(o)) for o in r[2:]]) + "\n")
    L += ["  <beam>", "    <type>PARALLEL</type>", "    <shape>CIRC</shape>", "    <profile>RANDOM</profile>",
          "    <range_distr>UNIFORM</range_distr>", f"    <params>{n_per_lambda} 0 {_num(radius)}</params>",
          "    <center>0 0 0</center>", f"    <range>{rng}</range>"]
    if n_lambda:
        L.append(f"    <nlambda>{int(n_lambda)}</nlambda>")
    L += ["  </beam>", "</scheme>", ""]
    with open(path, "w") as f:
        f.write("\n".join(L))


class LoadedScheme:
    """A scheme file read by the library (rtb_scheme_load): `surfaces` are
    rtb_surface structs (valid while this object lives), `beam` the <beam>
    element, `ranges` an (n, row_len) array, plus name / result_file /
    log_file / comments."""

    def __init__(self, path: str):
        L = ffi.load()
        L.rtb_scheme_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int)]
        L.rtb_scheme_surfaces.argtypes = [C.c_void_p, C.POINTER(C.POINTER(ffi.Surface)), C.POINTER(C.c_size_t)]
        L.rtb_scheme_text.argtypes = [C.c_void_p, C.c_int]
        L.rtb_scheme_text.restype = C.c_char_p
        L.rtb_scheme_get_beam.argtypes = [C.c_void_p, C.POINTER(ffi.SchemeBeam)]
        L.rtb_scheme_ranges.argtypes = [C.c_void_p, C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.c_size_t),
                                        C.POINTER(C.c_size_t)]
        L.rtb_scheme_free.argtypes = [C.c_void_p]
        self._L = L
        self.h = C.c_void_p()
        err = C.c_int(-1)
        self.status = L.rtb_scheme_load(path.encode(), C.byref(self.h), C.byref(err))
        self.scheme_error = err.value
        if self.status != ffi.OK:
            self.h = C.c_void_p()
            return
        p = C.POINTER(ffi.Surface)()
        n = C.c_size_t()
        ffi.check(L.rtb_scheme_surfaces(self.h, C.byref(p), C.byref(n)), "rtb_scheme_surfaces")
        self.surfaces = [p[i] for i in range(n.value)]
        for s in self.surfaces:
            s._owner = self
        self.beam = ffi.SchemeBeam()
        ffi.check(L.rtb_scheme_get_beam(self.h, C.byref(self.beam)), "rtb_scheme_get_beam")
        rp = C.POINTER(C.c_double)()
        nr, rl = C.c_size_t(), C.c_size_t()
        ffi.check(L.rtb_scheme_ranges(self.h, C.byref(rp), C.byref(nr), C.byref(rl)), "rtb_scheme_ranges")
        self.ranges = np.array([rp[i] for i in range(nr.value * rl.value)]).reshape(nr.value, rl.value)
        txt = lambda k: (L.rtb_scheme_text(self.h, k) or b"").decode()  # noqa: E731
        self.name, self.result_file, self.log_file = txt(0), txt(1), txt(2)
        self.comments = [txt(3 + k) for k in range(n.value)]
        L.rtb_scheme_qe_surfaces.argtypes = [C.c_void_p, C.POINTER(C.POINTER(ffi.QeSurface)),
                                             C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
        qp = C.POINTER(ffi.QeSurface)()
        nq, qerr = C.c_size_t(), C.c_int(-1)
        self.qe_status = L.rtb_scheme_qe_surfaces(self.h, C.byref(qp), C.byref(nq), C.byref(qerr))
        self.qe_error = qerr.value
        self.qe_array = (ffi.QeSurface * max(1, nq.value))()
        for i in range(nq.value):
            self.qe_array[i] = qp[i]          # tables still point into the scheme (kept alive by self)
        self.n_qe = nq.value

    def __del__(self):
        if getattr(self, "h", None):
            self._L.rtb_scheme_free(self.h)
            self.h = C.c_void_p()


def benchmark_scheme_files(out_dir: str) -> list[str]:
    """Write C0, C1 and C4 as scheme files (with their tables and C1's range
    file of one row per echelle order)."""
    import os
    os.makedirs(out_dir, exist_ok=True)
    c0 = os.path.join(out_dir, "c0_littrow_free.xml")
    write_xml(c0, littrow_free(), "C0 Littrow-free spectrograph", "c0", 20000, C0_RADIUS,
              [list(C0_LAMBDA)], n_lambda=C0_NLAMBDA)
    c1 = os.path.join(out_dir, "c1_echelle.xml")
    write_xml(c1, echelle(), "C1 cross-dispersed echelle", "c1", c1_rays_per_lambda(), C1_RADIUS,
              [[C1_LAMBDA[0], C1_LAMBDA[1], m, 1] for m in C1_ORDERS], n_lambda=C1_NLAMBDA)
    c4 = os.path.join(out_dir, "c4_littrow_free_flattener.xml")
    write_xml(c4, littrow_free_asphere(), "C4 Littrow-free spectrograph with an aspheric field flattener", "c4",
              156250, C0_RADIUS, [list(C4_LAMBDA)], n_lambda=C4_NLAMBDA)
    return [c0, c1, c4]


if __name__ == "__main__":
    import sys
    for p in benchmark_scheme_files(sys.argv[1] if len(sys.argv) > 1 else "."):
        print(p)
