// mixed.cuh -- device code of the fused mixed-precision trace kernel.
//
// Same per-ray algorithm as the plain engine (ray_fp64.cuh) with the
// precision of each step chosen for cost against its effect on the CCD
// position:
//   * ray state, transforms, intersection roots (the conic quadratic in a
//     cancellation-safe form; Newton for the even asphere from the base-conic
//     root and for the toric from the plane point, until a step falls below
//     1e-5 mm, the root then good to ~1e-12 mm), the grating equation and the
//     detector coordinate: FP64, contracted to FMA;
//   * every division and square root: a MUFU seed (rcp/rsqrt.approx.f64)
//     refined by one Newton step in FP64 (~2^-43 relative) instead of the
//     IEEE FP64 division and square root sequences of the plain engine; the
//     inverse of a Newton derivative from the seed alone; 1/c and
//     1/(grating constant) from the host;
//   * surface normals and their polynomial terms (the sqrt/div-heavy
//     derivatives of conic_derivs / toric_derivs, surface.cu:45-94): FP32
//     (from FP32 copies of the surface constants), promoted to FP64 before
//     they act on the direction cosines.  Their transverse components are
//     small, so the FP32 rounding moves a direction by ~1e-9 rad.
// Compiled with FMA contraction.  Accuracy is measured against the FP64
// oracle (median, p99.9 and max CCD error in um; target p99.9 <= 0.05 um).
// The surface code reads each surface's structure through a shape policy
// (shape.cuh): at run time in k_fused_mixed, fixed at compile time in the
// copies compiled for one scheme (jit.cpp).
#pragma once

#include "trace_common.cuh"
#include "ray_fp64.cuh"
#include "rowpipe.cuh"

namespace rtb {
namespace mx {

struct Ray {
    double X, Y, Z, cX, cY, cZ;
};

// Precision of the reciprocals and square roots.  Each comes from a MUFU seed
// (~2^-22 relative) and one Newton step, which leaves ~2^-43 relative: a
// ray parameter or distance of 1 m is then off by ~1e-10 mm, and a direction
// by ~1e-13 rad, five orders of magnitude below the 0.05 um (5e-5 mm) budget
// at the detector, whose error comes from the FP32 normals (~1e-8 rad).  A
// second step (full FP64 precision) would cost two more FP64 instructions per
// reciprocal and three per square root, ~70 per C1 ray.

// 1/x: rcp.approx.ftz.f64 seed and one Newton step (~2^-43 relative).
__device__ __forceinline__ double rcp(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

// 1/x to about 2^-22 (the seed alone): the inverse of a Newton derivative,
// whose error slows the convergence by that factor but does not move the root.
__device__ __forceinline__ double rcp_seed(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    return r;
}

// 1/sqrt(x): rsqrt.approx.f64 seed and `steps` Newton steps.
__device__ __forceinline__ double rsqrt_n(double x, int steps) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double h = 0.5 * x;
    for (int i = 0; i < steps; ++i) y = y * fma(-h * y, y, 1.5);
    return y;
}

// sqrt(x) ~2^-43 relative: s = x * rsqrt seed, then one Newton correction
// of the product, s + (x - s^2) / (2 sqrt x) with 1/sqrt x from the seed;
// NaN for x < 0, 0 for x == 0.
__device__ __forceinline__ double sqrt_(double x) {
    if (!(x > 0.0)) return (x == 0.0) ? 0.0 : __longlong_as_double(0x7ff8000000000000ll);
    const double y = rsqrt_n(x, 0);
    const double s = x * y;
    return fma(0.5 * y, fma(-s, s, x), s);
}

// Unit direction cosines: 1/|c| from the rsqrt seed and one Newton step.
__device__ __forceinline__ void normalize(Ray& r) {
    double s = fma(r.cX, r.cX, fma(r.cY, r.cY, r.cZ * r.cZ));
    double k = rsqrt_n(s, 1);
    r.cX *= k;
    r.cY *= k;
    r.cZ *= k;
}

template <class Sh>
__device__ __forceinline__ void transform(const DevSurface& s, Ray& r) {
    if (Sh::translate(s)) {
        r.X -= s.dist[0];
        r.Y -= s.dist[1];
        r.Z -= s.dist[2];
    }
    auto rot = [](double sA, double cA, double& v1, double& v2) {
        double e = fma(v1, cA, -v2 * sA);
        v2 = fma(v1, sA, v2 * cA);
        v1 = e;
    };
    const int rot_mask = Sh::rot_mask(s);
    if (rot_mask & 1) { rot(s.sinA[0], s.cosA[0], r.X, r.Z); rot(s.sinA[0], s.cosA[0], r.cX, r.cZ); }
    if (rot_mask & 2) { rot(s.sinA[1], s.cosA[1], r.Y, r.Z); rot(s.sinA[1], s.cosA[1], r.cY, r.cZ); }
    if (rot_mask & 4) { rot(s.sinA[2], s.cosA[2], r.X, r.Y); rot(s.sinA[2], s.cosA[2], r.cX, r.cY); }
}

// ---- surface normals in FP32 -------------------------------------------------

// (dF/dX, dF/dY) of the conic + even polynomial; dF/dZ = 1 (conic_derivs).
template <class Sh>
__device__ __forceinline__ void conic_normal(const DevSurface& s, double X, double Y, double& nx, double& ny) {
    float x = (float)X, y = (float)Y;
    float r2 = fmaf(x, x, y * y);
    float c = s.f_c, k1 = s.f_k1;
    float E = c * rsqrtf(fmaf(-k1 * c * c, r2, 1.0f));
    float sum = 0.0f, rr = 1.0f;
    const int N = Sh::n_poly(s);
    for (int i = 1; i <= N; ++i, rr *= r2) sum = fmaf(s.f_ipoly[i - 1], rr, sum);
    E = fmaf(2.0f, sum, E);
    nx = (double)(-E * x);
    ny = (double)(-E * y);
}

// (dF/dX, dF/dY, dF/dZ) of the toric surface (toric_derivs).
template <class Sh>
__device__ __forceinline__ void toric_normal(const DevSurface& s, double X, double Y, double Z, double& nx, double& ny,
                                             double& nz) {
    float y = (float)Y;
    float Y2 = y * y;
    float c = s.f_c, k1 = s.f_k1, cR = s.f_cR;
    float q = fmaf(-k1 * c * c, Y2, 1.0f);
    float rq = rsqrtf(q);
    float Fy = c * Y2 / (1.0f + q * rq);
    float sum = 0.0f, rr = Y2;
    const int N = Sh::n_poly(s);
    for (int i = 0; i < N; ++i, rr *= Y2) sum = fmaf(s.f_poly[i], rr, sum);
    Fy += sum;
    float dFy = c * y * rq;
    sum = 0.0f;
    rr = 1.0f;
    for (int i = 1; i <= N; ++i, rr *= Y2) sum = fmaf(s.f_ipoly[i - 1], rr, sum);
    dFy = fmaf(2.0f, sum, dFy);
    nx = (double)(-cR * (float)X);
    ny = (double)((cR * Fy - 1.0f) * dFy);
    nz = 1.0 - s.cR * Z;
}

template <class Sh>
__device__ __forceinline__ void normal(const DevSurface& s, const Ray& r, double& nx, double& ny, double& nz) {
    if (Sh::cls(s) == RTB_TORIC) {
        toric_normal<Sh>(s, r.X, r.Y, r.Z, nx, ny, nz);
    } else {
        conic_normal<Sh>(s, r.X, r.Y, nx, ny);
        nz = 1.0;
    }
}

// ---- intersections (FP64) ----------------------------------------------------

__device__ __forceinline__ bool plane_isect(Ray& r) {
    double s0 = -r.Z * rcp(r.cZ);
    if (s0 < 0.0) return false;
    r.X = fma(r.cX, s0, r.X);
    r.Y = fma(r.cY, s0, r.Y);
    r.Z = 0.0;
    return true;
}

// Paraboloid with the reference's linear root (surface.cu:183-213).
__device__ __forceinline__ bool paraboloid_isect(const DevSurface& s, Ray& r) {
    double ic = s.inv_c;
    double B = 2.0 * (fma(s.k1 * r.Z, r.cZ, fma(r.X, r.cX, r.Y * r.cY)) - r.cZ * ic);
    double C = fma(s.k1 * r.Z, r.Z, fma(r.X, r.X, r.Y * r.Y)) - 2.0 * r.Z * ic;
    double t = -C * rcp(B);
    if (t < 0.0) return false;
    r.X = fma(t, r.cX, r.X);
    r.Y = fma(t, r.cY, r.Y);
    r.Z = fma(t, r.cZ, r.Z);
    return true;
}

// Root of the base conic (c, k1) chosen as conic_intersection chooses it
// (surface.cu:240-244), evaluated without cancellation.  False if D < 0.
__device__ __forceinline__ bool conic_root(double c, double k1, double ic, const Ray& r, double& t) {
    double A = fma(k1 * r.cZ, r.cZ, fma(r.cX, r.cX, r.cY * r.cY));
    double B = 2.0 * (fma(k1 * r.Z, r.cZ, fma(r.X, r.cX, r.Y * r.cY)) - r.cZ * ic);
    double C = fma(k1 * r.Z, r.Z, fma(r.X, r.X, r.Y * r.Y)) - 2.0 * r.Z * ic;
    double D = fma(B, B, -4.0 * A * C);
    if (D < 0.0) return false;
    double sq = sqrt_(D);
    double q_pick = (c > 0) ? (-B - sq) : (-B + sq);
    double q_other = (c > 0) ? (-B + sq) : (-B - sq);
    // q_pick cancels when its two terms have opposite signs; then use
    // t = 2C / q_other (q_pick * q_other = 4AC).
    bool cancels = (c > 0) ? (B < 0) : (B > 0);
    t = cancels ? 2.0 * C * rcp(q_other) : q_pick * rcp(2.0 * A);
    return true;
}

__device__ __forceinline__ bool conic_isect(const DevSurface& s, Ray& r) {
    double t;
    if (!conic_root(s.c, s.k1, s.inv_c, r, t)) return false;
    r.X = fma(t, r.cX, r.X);
    r.Y = fma(t, r.cY, r.Y);
    r.Z = fma(t, r.cZ, r.Z);
    return true;
}

// Even asphere (iterative_conic_intersection / iterative_poly_intersection,
// surface.cu:257-333,497-561): the same surface and loss tests (plane point
// behind the ray, grazing |dF| < 1e-7), the root found differently.  With
// w = Z - P(r^2), P the even polynomial, the asphere is the base conic's
// quadric k1 w^2 + r^2 - 2 w / c = 0 on the branch the conic root selects, so
// Newton on G(t) = k1 w^2 + r^2 - 2 w / c (a polynomial in the ray parameter:
// no square root per step) from the base-conic root, the derivative's inverse
// taken from the reciprocal seed (rcp_seed).  Newton converges
// quadratically, the next correction being about |G''/2G'| dt^2 (< 1e-2 dt^2
// for these surfaces) plus the seed's 2^-22 dt, so the loop stops after a
// step below 1e-5 mm: the root is then good to ~1e-12 mm.  One step from the
// conic root for most rays; at most eight for rays that start far from the
// surface (far outside the aperture).
//
// Rays far outside the aperture take most of those steps, and their lanes
// hold the warp: a ray that within the slab sag_lo <= Z <= sag_hi (every
// surface point inside a circular aperture lies in it) stays outside the
// aperture's cylinder cannot meet the surface inside the aperture, so it is
// lost at the aperture without a root.  Returns 0 for a hit, 1 for a loss at
// the intersection, 2 for a loss at the aperture.
__device__ __forceinline__ bool misses_aperture(const DevSurface& s, const Ray& r) {
    if (r.cZ == 0.0) return false;
    const double iz = rcp(r.cZ);
    double ta = (s.sag_lo - r.Z) * iz, tb = (s.sag_hi - r.Z) * iz;
    if (ta > tb) {
        const double u = ta;
        ta = tb;
        tb = u;
    }
    const double px = r.X - s.center[0], py = r.Y - s.center[1];
    const double dd = fma(r.cX, r.cX, r.cY * r.cY);
    double t = (dd > 0.0) ? -fma(px, r.cX, py * r.cY) * rcp(dd) : ta;
    t = fmin(fmax(t, ta), tb);
    const double x = fma(t, r.cX, px), y = fma(t, r.cY, py);
    return fma(x, x, y * y) > s.size[0] * s.size[0] * (1.0 + 1e-9);
}

template <class Sh>
__device__ __forceinline__ int asphere_isect(const DevSurface& s, Ray& r) {
    double s0 = -r.Z * rcp(r.cZ);
    const bool poly_only = Sh::poly_only(s);
    if (poly_only ? !(s0 > 0) : !(s0 >= 0)) return 1;
    if (Sh::sag_cull(s) && misses_aperture(s, r)) return 2;
    double t = s0;
    double ic = 0.0;
    if (!poly_only) {
        double tc;
        if (conic_root(s.c, s.k1, s.inv_c, r, tc)) t = tc;
        ic = s.inv_c;
    }
    const int N = Sh::n_poly(s);
    double x = 0, y = 0;
    for (int it = 0; it < 8; ++it) {
        x = fma(t, r.cX, r.X);
        y = fma(t, r.cY, r.Y);
        const double z = fma(t, r.cZ, r.Z);
        const double r2 = fma(x, x, y * y);
        // P(r2) = r2 Q(r2), Q = a_1 + a_2 r2 + ... + a_N r2^(N-1) by Horner
        // with its derivative Q'; dP/dr2 = Q + r2 Q'
        double Q = 0.0, dQ = 0.0;
        for (int i = N; i >= 1; --i) {
            dQ = fma(dQ, r2, Q);
            Q = fma(Q, r2, s.poly[i - 1]);
        }
        const double P = Q * r2;
        const double dP = fma(r2, dQ, Q);
        const double dr2 = 2.0 * fma(x, r.cX, y * r.cY);  // d r2 / dt
        const double w = z - P;
        const double dw = fma(-dP, dr2, r.cZ);
        double G, dG;
        if (poly_only) {
            G = w;
            dG = dw;
        } else {
            G = fma(s.k1 * w, w, r2) - 2.0 * w * ic;
            dG = fma(2.0 * s.k1 * w, dw, dr2) - 2.0 * dw * ic;
        }
        const double dt = G * rcp_seed(dG);
        t -= dt;
        if (!(fabs(dt) >= 1e-5)) break;
    }
    if (!isfinite(t)) return 1;  // no root near the ray (far outside any aperture)
    x = fma(t, r.cX, r.X);
    y = fma(t, r.cY, r.Y);
    // the reference's grazing test on dF = cZ - E (x cX + y cY) at the root
    {
        const float xf = (float)x, yf = (float)y, c = s.f_c;
        const float r2 = fmaf(xf, xf, yf * yf);
        float E = 0.0f;
        if (!poly_only) {
            const float q = fmaf(-s.f_k1 * c * c, r2, 1.0f);
            E = (q > 0.0f) ? c * rsqrtf(q) : 0.0f;
        }
        float sum = 0.0f, rr = 1.0f;
        for (int i = 1; i <= N; ++i, rr *= r2) sum = fmaf(s.f_ipoly[i - 1], rr, sum);
        E = fmaf(2.0f, sum, E);
        const float dF = fmaf(-E, fmaf(xf, (float)r.cX, yf * (float)r.cY), (float)r.cZ);
        if (fabsf(dF) < (float)K_ITER_EPS) return 1;
    }
    r.X = x;
    r.Y = y;
    r.Z = fma(t, r.cZ, r.Z);
    return 0;
}

// Toric surface (iter_toric, surface.cu:359-410): the same function F of the
// reference (with its 1+k1c^2Y^2 unless RTB_FIX_TORIC_SIGN), solved by
// Newton from the Z=0 plane point with the analytic derivative (its FY' and
// its inverse from the reciprocal seed, rcp_seed)
//   dF/dt = cZ - FY' cY - cR (X cX + Z cZ - FY FY' cY),  FY' = c Y / s,
// s = sqrt(1 -+ k1 c^2 Y^2) (FY = c Y^2 / (1 + s) has this derivative for
// either sign), until a step falls below 1e-5 mm (quadratic convergence: the
// next correction, |F''/2F'| dt^2 plus the seed's 2^-22 dt, is ~1e-12 mm), at
// most six steps.  As in the reference, a
// ray is lost only when the plane point lies behind it.
__device__ __forceinline__ bool toric_isect(const DevSurface& s, uint32_t fixes, Ray& r) {
    const double sgn = (fixes & RTB_FIX_TORIC_SIGN) ? -1.0 : 1.0;
    double t = -r.Z * rcp(r.cZ);
    if (!(t >= 0)) return false;
    const double kc2 = sgn * s.k1 * s.c * s.c;
    for (int it = 0; it < 6; ++it) {
        double X = fma(t, r.cX, r.X), Y = fma(t, r.cY, r.Y), Z = fma(t, r.cZ, r.Z);
        double Y2 = Y * Y;
        double sq = sqrt_(fma(kc2, Y2, 1.0));
        double FY = s.c * Y2 * rcp(1.0 + sq);
        double dFY = s.c * Y * rcp_seed(sq);
        double F = Z - FY - 0.5 * s.cR * (fma(X, X, Z * Z) - FY * FY);
        double dF = r.cZ - dFY * r.cY - s.cR * (fma(X, r.cX, Z * r.cZ) - FY * dFY * r.cY);
        double dt = F * rcp_seed(dF);
        t -= dt;
        if (!(fabs(dt) >= 1e-5)) break;  // next correction ~|F''/2F'| dt^2 + 2^-22 dt ~ 1e-12 mm
    }
    r.X = fma(t, r.cX, r.X);
    r.Y = fma(t, r.cY, r.Y);
    r.Z = fma(t, r.cZ, r.Z);
    return true;
}

// 0: hit, 1: lost at the intersection, 2: lost at the aperture (known before the root).
template <class Sh>
__device__ __forceinline__ int intersect(const DevSurface& s, uint32_t fixes, Ray& r) {
    switch (Sh::kind(s)) {
        case IS_PLANE: return plane_isect(r) ? 0 : 1;
        case IS_PARABOLOID: return paraboloid_isect(s, r) ? 0 : 1;
        case IS_CONIC: return conic_isect(s, r) ? 0 : 1;
        case IS_ITER_POLY:
        case IS_ITER_CONIC: return asphere_isect<Sh>(s, r);
        case IS_TORIC: return toric_isect(s, fixes, r) ? 0 : 1;
        default: return 0;
    }
}

// ---- actions -------------------------------------------------------------------

// The actions take the surface normal (nx, ny, nz) at the ray's point,
// computed once per surface by action(); (0, 0, 1) on a plane.
__device__ __forceinline__ void reflect(double nx, double ny, double nz, Ray& r) {
    double a2 = 2.0 * fma(r.cX, nx, fma(r.cY, ny, r.cZ * nz)) * rcp(fma(nx, nx, fma(ny, ny, nz * nz)));
    r.cX = fma(-a2, nx, r.cX);
    r.cY = fma(-a2, ny, r.cY);
    r.cZ = fma(-a2, nz, r.cZ);
}

__device__ __forceinline__ bool refract(double mu, double nx, double ny, double nz, Ray& r) {
    double iG = rcp(fma(nx, nx, fma(ny, ny, nz * nz)));
    double a = mu * fma(r.cX, nx, fma(r.cY, ny, r.cZ * nz)) * iG;
    double b = fma(mu, mu, -1.0) * iG;
    double a2 = a * a;
    if (b > a2) return false;
    double G = -a + sqrt_(a2 - b);
    r.cX = fma(mu, r.cX, G * nx);
    r.cY = fma(mu, r.cY, G * ny);
    r.cZ = fma(mu, r.cZ, G * nz);
    return true;
}

// Grating equation (surface.cu:1247-1520) in FP64.
template <class Sh>
__device__ __forceinline__ bool diffract(const DevSurface& s, double mu, double L, double nx, double ny, double nz,
                                         Ray& r) {
    const bool trans = Sh::gr_type(s) == RTB_TRANSPARENT;
    const int cls = Sh::cls(s);
    if (cls == RTB_PLANE) {
        double a = trans ? mu * r.cZ : r.cZ;
        double b = trans ? fma(mu, mu, -1.0) + fma(L, L, -2.0 * mu * L * r.cX) : fma(L, L, -2.0 * L * r.cX);
        double a2 = a * a;
        if (b > a2) return false;
        double sq = sqrt_(a2 - b);
        if (trans) {
            r.cX = fma(mu, r.cX, -L);
            r.cY *= mu;
            r.cZ = fma(mu, r.cZ, -a + sq);
        } else {
            r.cX -= L;
            r.cZ += -a - sq;
        }
        return true;
    }
    // rule direction p = (u, v, w), as the reference builds it (including its
    // L^2+M+M for the toric, surface.cu:1438,1487)
    double den = (cls == RTB_TORIC) ? fma(ny, ny, nz + nz) : fma(ny, ny, 1.0);
    double G = nx * rcp(den);
    double u = rsqrt_n(fma(nx, G, 1.0), 1);
    double v = -ny * u * G;
    double w = (cls == RTB_TORIC) ? -nz * u * G : -u * G;
    double iG = rcp(fma(nx, nx, fma(ny, ny, nz * nz)));
    double kn = fma(r.cX, nx, fma(r.cY, ny, r.cZ * nz));
    double kp = fma(r.cX, u, fma(r.cY, v, r.cZ * w));
    double a, b;
    if (trans) {
        a = mu * kn * iG;
        b = (fma(mu, mu, -1.0) + fma(L, L, -2.0 * L * mu * kp)) * iG;
    } else {
        a = kn * iG;
        b = fma(L, L, -2.0 * L * kp) * iG;
    }
    double a2 = a * a;
    if (b > a2) return false;
    double sq = sqrt_(a2 - b);
    double g = trans ? -a + sq : -a - sq;
    double m = trans ? mu : 1.0;
    r.cX = fma(m, r.cX, fma(-L, u, g * nx));
    r.cY = fma(m, r.cY, fma(-L, v, g * ny));
    r.cZ = fma(m, r.cZ, fma(-L, w, g * nz));
    return true;
}

// Tabulated function with the divisions by the knot spacing replaced by a
// reciprocal.  A table on a uniform grid (invh = 1/spacing > 0) finds its
// interval directly, a non-uniform one by bisection; at a knot the spline
// formula returns y there to rounding, so no exact-knot branch is needed.
__device__ __forceinline__ bool table_eval(const double* tab, int n, double invh, double xval, double& out) {
    if (n == 1) {
        out = tab[1];
        return true;
    }
    const double* x = tab;
    const double* y = tab + n;
    const double* y2 = tab + 2 * n;
    if ((xval < x[0]) || (xval > x[n - 1])) return false;
    int il, ir;
    if (invh > 0.0) {
        il = (int)((xval - x[0]) * invh);
        il = il < 0 ? 0 : (il > n - 2 ? n - 2 : il);
        if (x[il] > xval && il > 0) --il;
        else if (x[il + 1] < xval && il < n - 2) ++il;
        ir = il + 1;
    } else {
        il = 0;
        ir = n;
        while ((ir - il) > 1) {
            int i = (il + ir) >> 1;
            if (x[i] > xval) ir = i; else il = i;
        }
        if (ir == n) {  // xval == x[n-1]
            il = n - 2;
            ir = n - 1;
        }
    }
    double h = x[ir] - x[il];
    double ih = rcp(h);
    double a = (x[ir] - xval) * ih;
    double b = (xval - x[il]) * ih;
    double cub = fma(fma(a, a * a, -a), y2[il], fma(b, b * b, -b) * y2[ir]);
    out = fma(a, y[il], fma(b, y[ir], cub * (h * h) * (1.0 / 6.0)));
    return true;
}

// The last table value a ray evaluated (a lens's glass is looked up by its
// front and its back surface at the same wavelength).
struct TableMemo {
    int off = -1;
    double v = 0.0;
};

__device__ __forceinline__ bool table_at(const double* knots, int off, int n, double invh, double lambda,
                                         TableMemo& m, double& out) {
    if (n == 1) {
        out = knots[off + 1];
        return true;
    }
    if (off == m.off) {
        out = m.v;
        return true;
    }
    if (!table_eval(knots + off, n, invh, lambda, out)) return false;
    m.off = off;
    m.v = out;
    return true;
}

// One site for each of the table lookups and the normal keeps the kernel's
// code small: it is bound by instruction fetch as much as by FP64 issue.
template <class Sh>
__device__ __forceinline__ int action(const DevSurface& s, const double* knots, long long order, double lambda,
                                      TableMemo& memo, Ray& r) {
    const int type = Sh::type(s), cls = Sh::cls(s), gr_type = Sh::gr_type(s);
    if (type == RTB_MIRROR && cls == RTB_PLANE) {
        r.cZ = -r.cZ;
        return 0;
    }
    double n1v = 1.0, n2v = 1.0;
    if (type == RTB_LENS || type == RTB_GRATING) {
        const int first = (type == RTB_LENS || gr_type == RTB_TRANSPARENT) ? 0 : 1;
#pragma unroll 1
        for (int t = first; t < 2; ++t) {
            double v;
            if (!table_at(knots, t ? s.n2_off : s.n1_off, t ? s.n2_n : s.n1_n, t ? s.n2_invh : s.n1_invh, lambda,
                          memo, v))
                return 2;
            if (t) n2v = v;
            else n1v = v;
        }
    }
    double nx = 0.0, ny = 0.0, nz = 1.0;
    if (cls != RTB_PLANE) normal<Sh>(s, r, nx, ny, nz);
    if (type == RTB_MIRROR) {
        reflect(nx, ny, nz, r);
        return 0;
    }
    const double in2 = rcp(n2v);
    if (type == RTB_LENS) return refract(n1v * in2, nx, ny, nz, r) ? 0 : 1;
    if (type == RTB_GRATING) {
        const double mu = (gr_type == RTB_TRANSPARENT) ? n1v * in2 : 0.0;
        const double L = (double)order * lambda * in2 * s.inv_gr;
        if (!diffract<Sh>(s, mu, L, nx, ny, nz, r)) return 1;
        // the reference's rule direction on a toric (L^2+M+M) is neither a
        // unit vector nor orthogonal to the normal, so the diffracted cosines
        // are not a unit vector: the Normalize after the action matters here
        if (cls == RTB_TORIC) normalize(r);
        return 0;
    }
    return 0;
}

}  // namespace mx

// One surface of the mixed engine on one ray: -1 survived, a stage >= 0 that
// lost it, -2 a wavelength outside a table.  The reference normalises the
// direction cosines after every transform and action (beam.cpp:527-571);
// rotations and the reflection, refraction and plane and conic grating
// formulas preserve a unit vector, so here the cosines are normalised when a
// ray is loaded and after a toric grating only.
template <class Sh = RtShape>
__device__ __forceinline__ int mx_surface(const DevSurface& s, int k, uint32_t fixes, const double* knots,
                                          const BeamCtx& bc, double lam, mx::TableMemo& memo, mx::Ray& r) {
    mx::transform<Sh>(s, r);
    if (!Sh::non_aux(s)) return -1;
    const int hit = mx::intersect<Sh>(s, fixes, r);
    if (hit == 1) return 3 * k;
    if (hit == 2) return 3 * k + 1;
    if (!f64::aperture_pass(Sh::type(s) == RTB_SHADE, Sh::shape(s), s.size, s.center, r.X, r.Y)) return 3 * k + 1;
    const long long order = (Sh::type(s) == RTB_GRATING) ? bc.order(s) : s.order;
    int a = mx::action<Sh>(s, knots, order, lam, memo, r);
    if (a == 2) return -2;
    if (a == 1) return 3 * k + 2;
    return -1;
}

// The surfaces of one ray in order, until one loses it.  RtSurfaces reads
// each surface's structure from the scheme; a kernel specialised to one
// scheme (jit.cpp) passes a policy whose run() calls mx_surface with each
// surface's FixedShape in turn.
struct RtSurfaces {
    __device__ __forceinline__ static void run(const DevScheme* sch, const double* knots, const BeamCtx& bc,
                                               double lam, mx::TableMemo& memo, mx::Ray& r, int& stage) {
        for (int k = 0; k < sch->n_surfaces && stage == -1; ++k)
            stage = mx_surface(sch->s[k], k, sch->fixes, knots, bc, lam, memo, r);
    }
};

// Fused mixed-precision trace: one ray per lane at a time, the whole scheme
// in registers, the scheme and knot tables in shared memory, a persistent
// grid whose warps take tiles of rpt rows of 32 rays (rowpipe.cuh).  Plans
// feed it Row64 blocks in tracing order through the row pipeline (each row's
// bulk copy in flight while the warp traces the row before); one-shot traces
// read the SoA arrays.  The kernels that run it (k_fused_mixed and the
// scheme-specialised ones) are launched with blocks of up to 512 threads and
// 64 registers a thread, which keeps 32 warps resident per SM and hides the
// FP64 dependency chains better than more registers would (C1: 11.5 ms per
// step at 64 registers, 13.0 at 80, 16.1 at 96; below 64 the spills cost
// more).
template <class Surfaces>
__device__ __forceinline__ void fused_mixed(const DevScheme* __restrict__ g_sch, const double* knots,
                                            const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                            unsigned long long* counts, unsigned* err, int state_out,
                                            FrameArgs frame, TileSched ts) {
    const double* s_knots;
    const DevScheme* sch = stage_scheme(g_sch, knots, s_knots);
    const int n_stages = 3 * sch->n_surfaces;
    RowLoop rows(ts, in.n, warp_row_buffer<Row64>(sch->n_knots), (unsigned)sizeof(Row64), err);
    const int lane = threadIdx.x & 31;
    BeamCursor cur;
    while (rows.begin()) {
        const size_t slot = rows.slot();
        const bool valid = slot < in.n;
        // the ray's index, read only when its results go there; its beam: the
        // beam of its slot in a plan's (beam-major) tracing order
        const size_t i = (ts.order && valid && !(rows.packed && ts.out_by_slot)) ? (size_t)ts.order[slot] : slot;
        const size_t oi = ts.out_by_slot ? slot : i;
        const size_t bi = rows.packed ? slot : i;
        mx::Ray r{0, 0, 0, 0, 0, 0};
        double lam = 0.0;
        char f = 0;
        if (rows.packed) {
            const Row64& w = rows.row<Row64>();
            f = w.flag[lane];
            r = mx::Ray{w.X[lane], w.Y[lane], w.Z[lane], w.cX[lane], w.cY[lane], w.cZ[lane]};
            lam = w.lambda[lane];
        } else if (valid) {
            const size_t ri = ts.in_by_slot ? slot : i;
            f = in.flag[ri];
            if (f == 1) {
                r = mx::Ray{in.X[ri], in.Y[ri], in.Z[ri], in.cX[ri], in.cY[ri], in.cZ[ri]};
                lam = in.lambda[ri];
            }
        }
        rows.prefetch();
        bool ev = false, good = false;
        int key = 0;
        double outX = 0, outY = 0;
        int b = 0;
        if (valid && f == 1) {
            b = cur.at(beams, n_beams, bi);
            const BeamCtx& bc = cur.ctx;
            if (!rows.packed) mx::normalize(r);  // row blocks hold normalised cosines
            mx::TableMemo memo;
            int stage = -1;
            Surfaces::run(sch, s_knots, bc, lam, memo, r, stage);
            if (stage == -2) atomicOr(err, DEV_ERR_OUT_OF_RANGE);
            if (stage >= 0) {
                ev = true;
                out.flag[oi] = 0;
                out.lost_stage[oi] = (uint8_t)stage;
                key = b * (n_stages + 1) + stage;
            } else if (stage == -1) {
                ev = good = true;
                key = b * (n_stages + 1) + n_stages;
                if (rows.packed || in.flag != out.flag) {
                    out.flag[oi] = 1;
                    out.lost_stage[oi] = RTB_NOT_LOST;
                }
            }
            if (stage != -2) {
                out.X[oi] = r.X;
                out.Y[oi] = r.Y;
                if (state_out) {
                    out.Z[oi] = r.Z;
                    out.cX[oi] = r.cX;
                    out.cY[oi] = r.cY;
                    out.cZ[oi] = r.cZ;
                }
            }
            outX = r.X;
            outY = r.Y;
        } else if (valid && (rows.packed || in.flag != out.flag)) {
            out.flag[oi] = f;
        }
        count_event(ev, key, counts);
        if (frame.counts) frame_add<false>(good, outX, outY, frame);
    }
}

}  // namespace rtb
