// ray_rev.cuh -- reverse-mode derivatives of one surface of the plain FP64
// engine.
//
// surface_rev recomputes a surface on one ray from the ray's state at the
// surface's input (transform, normalise, and for a non-Aux surface the
// intersection, action and second normalisation, with the plain engine's
// functions and hence its values and branches), then carries the adjoint of
// the output state back through each stage in reverse order: the adjoint of
// the input state and of the surface's differentiable constants (curvature,
// conic constant, polynomial coefficients, toric radius, grating constant,
// distances, rotation sines and cosines).  One recomputation and one reverse
// sweep give every direction at once, where the forward-mode dual numbers of
// ray_ad.cuh need one pass per few directions.
//
// Each stage's adjoint is the transpose of the derivative ray_ad.cuh's dual
// numbers compute for the same expression, so the two agree to rounding:
//  * roots of iterations (asphere Newton, toric Steffensen) move with the
//    inputs as -F_inputs / F_t at the point the iteration returns (implicit
//    function theorem), F the surface function along the ray;
//  * the normalisation's derivative is that of c / |c|;
//  * a rotation or translation the plain engine skips (zero angle or
//    distance) is the identity, whose derivative in its angle or distance is
//    still taken.
//
// The translation unit is compiled with --fmad=false (the recomputed values
// are the plain engine's bits).
#pragma once

#include "ray_ad.cuh"
#include "ray_fp64.cuh"
#include "shape.cuh"

namespace rtb {
namespace rv {

// Reciprocal and reciprocal square root for the derivative arithmetic (the
// values the recomputation follows keep the plain engine's IEEE operations):
// the hardware seed refined by Newton steps (two for 1/x, x (2 - x y); two
// for 1/sqrt(x), y (3/2 - x y^2 / 2)), to about an ulp, in place of the
// IEEE division and square-root sequences.
__device__ __forceinline__ double rcp(double x) { return ad::tangent_rcp(x); }
__device__ __forceinline__ double rsqrt(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = 0.5 * x;
    y = y * fma(-h * y, y, 1.5);
    return y * fma(-h * y, y, 1.5);
}

// Adjoints of the ray state.
struct RayA {
    double X, Y, Z, cX, cY, cZ;
};

// Adjoints of one surface's differentiable constants (DevSurface fields).
struct SurfA {
    double c, k1, cR, gr;
    double poly[RTB_MAX_POLY];
    double dist[3], sA[3], cA[3];
};

__device__ __forceinline__ void clear(SurfA& p) {
    p.c = p.k1 = p.cR = p.gr = 0.0;
#pragma unroll
    for (int i = 0; i < RTB_MAX_POLY; ++i) p.poly[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) p.dist[i] = p.sA[i] = p.cA[i] = 0.0;
}

// ---- transform and normalisation --------------------------------------------

// (v1, v2) -> (v1 cA - v2 sA, v1 sA + v2 cA), the same for (w1, w2).  Inputs
// v, w; in: the adjoints of the outputs; out: those of the inputs.
__device__ __forceinline__ void rotate_pair_rev(double sA, double cA, double v1, double v2, double w1, double w2,
                                                double& av1, double& av2, double& aw1, double& aw2, double& asA,
                                                double& acA) {
    asA += -av1 * v2 + av2 * v1 - aw1 * w2 + aw2 * w1;
    acA += av1 * v1 + av2 * v2 + aw1 * w1 + aw2 * w2;
    double e = av1 * cA + av2 * sA;
    av2 = -av1 * sA + av2 * cA;
    av1 = e;
    e = aw1 * cA + aw2 * sA;
    aw2 = -aw1 * sA + aw2 * cA;
    aw1 = e;
}

// beam_transform (translation, then rotations about y, x, z) from the input
// state r0.  A rotation the engine skips has sinA = 0, cosA = 1: applying it
// leaves the values as they are.
__device__ __forceinline__ void transform_rev(const DevSurface& s, const f64::Ray& r0, RayA& a, SurfA& p) {
    f64::Ray ra = r0;
    ra.X -= s.dist[0];
    ra.Y -= s.dist[1];
    ra.Z -= s.dist[2];
    f64::Ray rb = ra;
    f64::rotate_pair(s.sinA[0], s.cosA[0], rb.X, rb.Z, rb.cX, rb.cZ);
    f64::Ray rc = rb;
    f64::rotate_pair(s.sinA[1], s.cosA[1], rc.Y, rc.Z, rc.cY, rc.cZ);
    rotate_pair_rev(s.sinA[2], s.cosA[2], rc.X, rc.Y, rc.cX, rc.cY, a.X, a.Y, a.cX, a.cY, p.sA[2], p.cA[2]);
    rotate_pair_rev(s.sinA[1], s.cosA[1], rb.Y, rb.Z, rb.cY, rb.cZ, a.Y, a.Z, a.cY, a.cZ, p.sA[1], p.cA[1]);
    rotate_pair_rev(s.sinA[0], s.cosA[0], ra.X, ra.Z, ra.cX, ra.cZ, a.X, a.Z, a.cX, a.cZ, p.sA[0], p.cA[0]);
    p.dist[0] -= a.X;
    p.dist[1] -= a.Y;
    p.dist[2] -= a.Z;
}

// c -> c / |c| at the pre-normalisation cosines c: the adjoint of c is the
// output adjoint's component orthogonal to the unit vector, over |c| (the
// derivative of Beam::Normalize's formula, which computes |c|).
__device__ __forceinline__ void normalize_rev(double cX, double cY, double cZ, RayA& a) {
    const double in = rsqrt(fma(cX, cX, fma(cY, cY, cZ * cZ)));
    const double uX = cX * in, uY = cY * in, uZ = cZ * in;
    const double d = a.cX * uX + a.cY * uY + a.cZ * uZ;
    a.cX = (a.cX - d * uX) * in;
    a.cY = (a.cY - d * uY) * in;
    a.cZ = (a.cZ - d * uZ) * in;
}

// ---- surface slopes ------------------------------------------------------------

// conic_derivs: dFdX = -E X, dFdY = -E Y with
// E = c / w + 2 sum_{i=1..n} i a_i r2^(i-1), w = sqrt(1 - k1 c^2 r2).
// In: the adjoints gX, gY of dFdX, dFdY.
template <class Sh = RtShape>
__device__ __forceinline__ void conic_derivs_rev(const DevSurface& s, double X, double Y, double gX, double gY,
                                                 RayA& a, SurfA& p) {
    const int n = Sh::n_poly(s);
    const double r2 = X * X + Y * Y;
    const double iw = rsqrt(1.0 - s.k1 * s.c * s.c * r2);
    const double iw3 = iw * iw * iw;
    const double gE = -(gX * X + gY * Y);
    double E = s.c * iw, dE = 0.5 * s.k1 * s.c * s.c * s.c * iw3;  // E and dE/dr2
    double rr = 1.0, rm = 0.0;                                       // r2^(i-1), r2^(i-2)
#pragma unroll
    for (int i = 1; i <= RTB_MAX_POLY; ++i) {
        if (i > n) break;
        E += 2.0 * i * s.poly[i - 1] * rr;
        dE += 2.0 * i * (i - 1) * s.poly[i - 1] * rm;
        p.poly[i - 1] += gE * 2.0 * i * rr;
        rm = rr;
        rr *= r2;
    }
    p.c += gE * (iw + s.k1 * s.c * s.c * r2 * iw3);
    p.k1 += gE * 0.5 * s.c * s.c * s.c * r2 * iw3;
    const double gr2 = gE * dE;
    a.X += -gX * E + 2.0 * X * gr2;
    a.Y += -gY * E + 2.0 * Y * gr2;
}

// toric_derivs: dFdX = -cR X, dFdY = (cR Fy - 1) dFy, dFdZ = 1 - cR Z with
// Fy = c Y2 / (1 + w) + sum_i a_i Y2^(i+1), dFy = c Y / w + 2 sum_{i=1..n} i a_i Y2^(i-1),
// w = sqrt(1 - k1 c^2 Y2).  In: the adjoints gX, gY, gZ of dFdX, dFdY, dFdZ.
template <class Sh = RtShape>
__device__ __forceinline__ void toric_derivs_rev(const DevSurface& s, double X, double Y, double Z, double gX,
                                                 double gY, double gZ, RayA& a, SurfA& p) {
    const int n = Sh::n_poly(s);
    const double c = s.c, k1 = s.k1, Y2 = Y * Y;
    const double q = 1.0 - k1 * c * c * Y2;
    const double iw = rsqrt(q), w = q * iw, iw3 = iw * iw * iw, iden = rcp(1.0 + w), iden2 = iden * iden;
    double Fy = c * Y2 * iden, dFy = c * Y * iw;
    {
        double rr = Y2, rq = 1.0;
#pragma unroll
        for (int i = 0; i < RTB_MAX_POLY; ++i) {
            if (i >= n) break;
            Fy += s.poly[i] * rr;
            dFy += 2.0 * (i + 1) * s.poly[i] * rq;
            rr *= Y2;
            rq *= Y2;
        }
    }
    p.cR += -gX * X + gY * Fy * dFy - gZ * Z;
    a.X += -gX * s.cR;
    a.Z += -gZ * s.cR;
    const double gFy = gY * s.cR * dFy;        // adjoint of Fy
    const double gdFy = gY * (s.cR * Fy - 1.0);  // adjoint of dFy
    // conic parts: Fy0 = c Y2 / (1 + w), dFy0 = c Y / w
    double dY2 = gFy * (c * iden + 0.5 * k1 * c * c * c * Y2 * iw * iden2) + gdFy * 0.5 * k1 * c * c * c * Y * iw3;
    p.c += gFy * (Y2 * iden + k1 * c * c * Y2 * Y2 * iw * iden2) + gdFy * (Y * iw + k1 * c * c * Y * Y2 * iw3);
    p.k1 += gFy * 0.5 * c * c * c * Y2 * Y2 * iw * iden2 + gdFy * 0.5 * c * c * c * Y * Y2 * iw3;
    {
        double rq = 1.0, rm = 0.0;  // Y2^i, Y2^(i-1)
#pragma unroll
        for (int i = 0; i < RTB_MAX_POLY; ++i) {
            if (i >= n) break;
            dY2 += gFy * (i + 1) * s.poly[i] * rq + gdFy * 2.0 * (i + 1) * i * s.poly[i] * rm;
            p.poly[i] += gFy * rq * Y2 + gdFy * 2.0 * (i + 1) * rq;
            rm = rq;
            rq *= Y2;
        }
    }
    a.Y += 2.0 * Y * dY2 + gdFy * c * iw;
}

// The slopes of a conic (dFdZ = 1) or toric surface at (X, Y, Z).
template <class Sh = RtShape>
__device__ __forceinline__ void slopes(const DevSurface& s, bool tor, double X, double Y, double Z, double& dX,
                                       double& dY, double& dZ) {
    if (tor) {
        f64::toric_derivs<Sh>(s, X, Y, Z, dX, dY, dZ);
    } else {
        f64::conic_derivs<Sh>(s, X, Y, dX, dY);
        dZ = 1.0;
    }
}

template <class Sh = RtShape>
__device__ __forceinline__ void slopes_rev(const DevSurface& s, bool tor, double X, double Y, double Z, double gX,
                                           double gY, double gZ, RayA& a, SurfA& p) {
    if (tor) toric_derivs_rev<Sh>(s, X, Y, Z, gX, gY, gZ, a, p);
    else conic_derivs_rev<Sh>(s, X, Y, gX, gY, a, p);
}

// ---- intersections -----------------------------------------------------------

// The point moves along the ray: P' = P + t c.  Passes the position adjoint
// through, adds t * (position adjoint) to the cosines' and returns the
// adjoint of t.
__device__ __forceinline__ double along_rev(const f64::Ray& r, double t, RayA& a) {
    const double gt = a.X * r.cX + a.Y * r.cY + a.Z * r.cZ;
    a.cX += a.X * t;
    a.cY += a.Y * t;
    a.cZ += a.Z * t;
    return gt;
}

// B = 2 (k1 Z cZ + X cX + Y cY - cZ / c), C = k1 Z^2 + X^2 + Y^2 - 2 Z / c.
__device__ __forceinline__ void quadric_BC_rev(const DevSurface& s, const f64::Ray& r, double gB, double gC, RayA& a,
                                               SurfA& p) {
    const double b2 = 2.0 * gB, ic = s.inv_c;
    p.k1 += b2 * r.Z * r.cZ + gC * r.Z * r.Z;
    p.c += (b2 * r.cZ + gC * 2.0 * r.Z) * ic * ic;
    a.X += b2 * r.cX + 2.0 * gC * r.X;
    a.Y += b2 * r.cY + 2.0 * gC * r.Y;
    a.Z += b2 * s.k1 * r.cZ + gC * (2.0 * s.k1 * r.Z - 2.0 * ic);
    a.cX += b2 * r.X;
    a.cY += b2 * r.Y;
    a.cZ += b2 * (s.k1 * r.Z - ic);
}

// Asphere surface function F = Z - sag(r2) - sum_i a_i r2^(i+1) at P = r + t c
// (t held), sag = c r2 / (1 + w), w = sqrt(1 - k1 c^2 r2); gF its adjoint.
template <class Sh = RtShape>
__device__ __forceinline__ void asphere_F_rev(const DevSurface& s, bool poly_only, const f64::Ray& r, double t,
                                              double gF, RayA& a, SurfA& p) {
    const double PX = r.X + t * r.cX, PY = r.Y + t * r.cY;
    const double r2 = PX * PX + PY * PY;
    double dsag = 0.0;  // d(sag + poly)/dr2
    if (!poly_only) {
        const double c = s.c, k1 = s.k1;
        const double q = 1.0 - k1 * c * c * r2;
        const double iw = rsqrt(q), w = q * iw, iden = rcp(1.0 + w), iden2 = iden * iden;
        dsag = c * iden + 0.5 * k1 * c * c * c * r2 * iw * iden2;
        p.c += -gF * (r2 * iden + k1 * c * c * r2 * r2 * iw * iden2);
        p.k1 += -gF * 0.5 * c * c * c * r2 * r2 * iw * iden2;
    }
    double rq = 1.0;  // r2^i
#pragma unroll
    for (int i = 0; i < RTB_MAX_POLY; ++i) {
        if (i >= Sh::n_poly(s)) break;
        dsag += (i + 1) * s.poly[i] * rq;
        p.poly[i] += -gF * rq * r2;
        rq *= r2;
    }
    const double gr2 = -gF * dsag;
    const double gPX = 2.0 * gr2 * PX, gPY = 2.0 * gr2 * PY, gPZ = gF;
    a.X += gPX;
    a.Y += gPY;
    a.Z += gPZ;
    a.cX += gPX * t;
    a.cY += gPY * t;
    a.cZ += gPZ * t;
}

// Toric surface function F = Z - FY - cR/2 (X^2 + Z^2 - FY^2) at P = r + t c,
// FY = c Y2 / (1 + q), q = sqrt(1 - kk c^2 Y2), kk = k1 with the sign fix
// and -k1 without it (toric_func).
__device__ __forceinline__ void toric_F_rev(const DevSurface& s, bool fix_sign, const f64::Ray& r, double t,
                                            double gF, RayA& a, SurfA& p) {
    const double PX = r.X + t * r.cX, PY = r.Y + t * r.cY, PZ = r.Z + t * r.cZ;
    const double c = s.c, kk = fix_sign ? s.k1 : -s.k1, Y2 = PY * PY;
    const double qq = 1.0 - kk * c * c * Y2;
    const double iq = rsqrt(qq), q = qq * iq, iden = rcp(1.0 + q), iden2 = iden * iden;
    const double FY = c * Y2 * iden;
    p.cR += gF * -0.5 * (PX * PX + PZ * PZ - FY * FY);
    const double gFY = gF * (s.cR * FY - 1.0);
    const double gY2 = gFY * (c * iden + 0.5 * kk * c * c * c * Y2 * iq * iden2);
    p.c += gFY * (Y2 * iden + kk * c * c * Y2 * Y2 * iq * iden2);
    const double dk = gFY * 0.5 * c * c * c * Y2 * Y2 * iq * iden2;
    p.k1 += fix_sign ? dk : -dk;
    const double gPX = gF * -s.cR * PX, gPY = 2.0 * gY2 * PY, gPZ = gF * (1.0 - s.cR * PZ);
    a.X += gPX;
    a.Y += gPY;
    a.Z += gPZ;
    a.cX += gPX * t;
    a.cY += gPY * t;
    a.cZ += gPZ * t;
}

// dF/dt along the ray at the reported point (the value ray_ad.cuh divides by).
template <class Sh = RtShape>
__device__ __forceinline__ double asphere_Ft(const DevSurface& s, bool poly_only, const f64::Ray& r, double t) {
    const double X = r.X + t * r.cX, Y = r.Y + t * r.cY;
    const double r2 = X * X + Y * Y;
    double E = 0.0;
    if (!poly_only) E = s.c * rsqrt(1.0 - s.k1 * s.c * s.c * r2);
    double sum = 0.0, rr = 1.0;
    for (int i = 1; i <= Sh::n_poly(s); ++i, rr *= r2) sum += (double)i * s.poly[i - 1] * rr;
    E += 2.0 * sum;
    return r.cZ - E * (X * r.cX + Y * r.cY);
}

__device__ __forceinline__ double toric_Ft(const DevSurface& s, bool fix_sign, const f64::Ray& r, double t) {
    const double X = r.X + t * r.cX, Y = r.Y + t * r.cY, Z = r.Z + t * r.cZ;
    const double sg = fix_sign ? -1.0 : 1.0;
    const double Y2 = Y * Y;
    const double qq = 1.0 + sg * s.k1 * s.c * s.c * Y2;
    const double iq = rsqrt(qq), q = qq * iq;
    const double FY = s.c * Y2 * rcp(1.0 + q), dFY = s.c * Y * iq;
    return r.cZ - dFY * r.cY - s.cR * (X * r.cX + Z * r.cZ - FY * dFY * r.cY);
}

// The intersection on the values, as f64::intersect computes it; t: the ray
// parameter of the reported point for the iterative kinds.
template <class Sh = RtShape>
__device__ __forceinline__ bool isect_fwd(const DevSurface& s, uint32_t fixes, f64::Ray& r, double& t) {
    t = 0.0;
    switch (Sh::kind(s)) {
        case IS_ITER_POLY:
        case IS_ITER_CONIC: {
            const double s0 = -r.Z / r.cZ;
            double s1;
            if (!ad::asphere_values(s, r, Sh::kind(s) == IS_ITER_POLY, (fixes & RTB_FIX_ASPHERE_ROOT) != 0, s1))
                return false;
            t = s1 + s0;
            r.X = r.X + t * r.cX;  // iterative_*_intersection's Xi, Yi, Zi
            r.Y = r.Y + t * r.cY;
            r.Z = s1 * r.cZ;
            return true;
        }
        case IS_TORIC: {
            if (!ad::toric_values(s, fixes, r, t)) return false;
            r.X += t * r.cX;
            r.Y += t * r.cY;
            r.Z += t * r.cZ;
            return true;
        }
        default: return f64::intersect<Sh>(s, fixes, r);
    }
}

// r: the state before the intersection; in: the adjoint after it.
template <class Sh = RtShape>
__device__ __forceinline__ void isect_rev(const DevSurface& s, uint32_t fixes, const f64::Ray& r, double t, RayA& a,
                                          SurfA& p) {
    switch (Sh::kind(s)) {
        case IS_PLANE: {
            const double icZ = rcp(r.cZ);
            const double s0 = -r.Z * icZ;
            const double g0 = a.X * r.cX + a.Y * r.cY;  // Z' = 0 carries nothing
            a.cX += a.X * s0;
            a.cY += a.Y * s0;
            a.Z = -g0 * icZ;
            a.cZ += -g0 * s0 * icZ;
            return;
        }
        case IS_PARABOLOID: {
            const double B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ * s.inv_c);
            const double C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z * s.inv_c;
            const double iB = rcp(B);
            const double tt = -C * iB;
            const double gt = along_rev(r, tt, a);
            quadric_BC_rev(s, r, -gt * tt * iB, -gt * iB, a, p);
            return;
        }
        case IS_CONIC: {
            const double A = s.k1 * r.cZ * r.cZ + r.cX * r.cX + r.cY * r.cY;
            const double B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ * s.inv_c);
            const double C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z * s.inv_c;
            const double D = B * B - 4.0 * A * C;
            const double iq = rsqrt(D), q = D * iq, iA = rcp(A);
            const double sg = (s.c > 0) ? -1.0 : 1.0;
            const double tt = (-B + sg * q) * 0.5 * iA;
            const double gt = along_rev(r, tt, a);
            const double gN = gt * 0.5 * iA;
            double gA = -gt * tt * iA;
            const double gD = sg * gN * 0.5 * iq;
            const double gB = -gN + 2.0 * B * gD;
            gA += -4.0 * C * gD;
            const double gC = -4.0 * A * gD;
            p.k1 += gA * r.cZ * r.cZ;
            a.cX += 2.0 * gA * r.cX;
            a.cY += 2.0 * gA * r.cY;
            a.cZ += 2.0 * gA * s.k1 * r.cZ;
            quadric_BC_rev(s, r, gB, gC, a, p);
            return;
        }
        case IS_ITER_POLY:
        case IS_ITER_CONIC: {
            const bool po = Sh::kind(s) == IS_ITER_POLY;
            const double gt = along_rev(r, t, a);
            asphere_F_rev<Sh>(s, po, r, t, -gt * rcp(asphere_Ft<Sh>(s, po, r, t)), a, p);
            return;
        }
        case IS_TORIC: {
            const bool fs = (fixes & RTB_FIX_TORIC_SIGN) != 0;
            const double gt = along_rev(r, t, a);
            toric_F_rev(s, fs, r, t, -gt * rcp(toric_Ft(s, fs, r, t)), a, p);
            return;
        }
        default: return;
    }
}

// ---- actions -------------------------------------------------------------------

// The refractive-index ratio and grating term of the action, as f64::action
// computes them.  False where a table is out of range.
template <class Sh = RtShape>
__device__ __forceinline__ bool action_consts(const DevSurface& s, const double* knots, long long order,
                                              double lambda, double& mu, double& L) {
    mu = 0.0;
    L = 0.0;
    if (Sh::type(s) == RTB_LENS) {
        double a, b;
        if (!f64::table_eval(knots + s.n1_off, s.n1_n, lambda, a) || !f64::table_eval(knots + s.n2_off, s.n2_n, lambda, b))
            return false;
        mu = a;
        mu /= b;
    } else if (Sh::type(s) == RTB_GRATING) {
        double n2v;
        if (!f64::table_eval(knots + s.n2_off, s.n2_n, lambda, n2v)) return false;
        if (Sh::gr_type(s) == RTB_TRANSPARENT) {
            double n1v;
            if (!f64::table_eval(knots + s.n1_off, s.n1_n, lambda, n1v)) return false;
            mu = n1v;
            mu /= n2v;
        }
        L = (double)order * lambda / n2v / s.gr_const;
    }
    return true;
}

template <class Sh = RtShape>
__device__ __forceinline__ bool action_fwd(const DevSurface& s, double mu, double L, f64::Ray& r) {
    if (Sh::type(s) == RTB_MIRROR) {
        f64::reflect<Sh>(s, r);
        return true;
    }
    if (Sh::type(s) == RTB_LENS) return f64::refract<Sh>(s, mu, r);
    if (Sh::type(s) == RTB_GRATING) return f64::diffract<Sh>(s, mu, L, r);
    return true;
}

// Reflection about the curved surface's normal: c' = c - a2 dF,
// a2 = 2 (c . dF) / |dF|^2.
template <class Sh = RtShape>
__device__ __forceinline__ void reflect_rev(const DevSurface& s, bool tor, const f64::Ray& r, RayA& a, SurfA& p) {
    double dX, dY, dZ;
    slopes<Sh>(s, tor, r.X, r.Y, r.Z, dX, dY, dZ);
    const double num = r.cX * dX + r.cY * dY + r.cZ * dZ;
    const double den = dX * dX + dY * dY + dZ * dZ;
    const double iden = rcp(den);
    const double a2 = 2.0 * num * iden;
    const double ga2 = -(a.cX * dX + a.cY * dY + a.cZ * dZ);
    double gX = -a.cX * a2, gY = -a.cY * a2, gZ = -a.cZ * a2;
    const double gn = 2.0 * ga2 * iden, gden = -ga2 * a2 * iden;
    a.cX += gn * dX;
    a.cY += gn * dY;
    a.cZ += gn * dZ;
    gX += gn * r.cX + 2.0 * gden * dX;
    gY += gn * r.cY + 2.0 * gden * dY;
    gZ += gn * r.cZ + 2.0 * gden * dZ;
    slopes_rev<Sh>(s, tor, r.X, r.Y, r.Z, gX, gY, gZ, a, p);
}

// Refraction at a curved surface: G0 = |dF|^2, a = mu (c . dF) / G0,
// b = (mu^2 - 1) / G0, G = -a + sqrt(a^2 - b), c' = mu c + G dF.
template <class Sh = RtShape>
__device__ __forceinline__ void refract_rev(const DevSurface& s, bool tor, double mu, const f64::Ray& r, RayA& a,
                                            SurfA& p) {
    double dX, dY, dZ;
    slopes<Sh>(s, tor, r.X, r.Y, r.Z, dX, dY, dZ);
    const double G0 = dX * dX + dY * dY + dZ * dZ;
    const double num = r.cX * dX + r.cY * dY + r.cZ * dZ;
    const double iG0 = rcp(G0);
    const double av = mu * num * iG0, bv = (mu * mu - 1.0) * iG0;
    const double d2 = av * av - bv, isq = rsqrt(d2), sq = d2 * isq;
    const double G = -av + sq;
    const double gG = a.cX * dX + a.cY * dY + a.cZ * dZ;
    double gX = a.cX * G, gY = a.cY * G, gZ = a.cZ * G;
    a.cX *= mu;
    a.cY *= mu;
    a.cZ *= mu;
    const double ga = -gG + gG * av * isq, gb = -gG * 0.5 * isq;
    const double gG0 = -(gb * bv + ga * av) * iG0;
    const double gn = ga * mu * iG0;
    a.cX += gn * dX;
    a.cY += gn * dY;
    a.cZ += gn * dZ;
    gX += gn * r.cX + 2.0 * gG0 * dX;
    gY += gn * r.cY + 2.0 * gG0 * dY;
    gZ += gn * r.cZ + 2.0 * gG0 * dZ;
    slopes_rev<Sh>(s, tor, r.X, r.Y, r.Z, gX, gY, gZ, a, p);
}

// Diffraction at a curved grating (transparent: m = mu, K = mu^2 - 1, sign +;
// reflective: m = 1, K = 0, sign -):
// g1 = dFdX / den1 (den1 = dFdY^2 + 1, or dFdY^2 + 2 dFdZ on a toric),
// u = 1 / sqrt(1 + dFdX g1), v = -dFdY u g1, w = -u g1 (toric: -dFdZ u g1),
// a = m (c . dF) / G0, b = (K + L^2 - 2 L m (c . uvw)) / G0,
// G = -a + sign sqrt(a^2 - b), c' = m c - L uvw + G dF.  Returns the
// adjoint of L.
template <class Sh = RtShape>
__device__ __forceinline__ double diffract_curved_rev(const DevSurface& s, bool tor, bool trans, double mu, double L,
                                                      const f64::Ray& r, RayA& a, SurfA& p) {
    double dX, dY, dZ;
    slopes<Sh>(s, tor, r.X, r.Y, r.Z, dX, dY, dZ);
    const double m = trans ? mu : 1.0, K = trans ? mu * mu - 1.0 : 0.0, sg = trans ? 1.0 : -1.0;
    const double den1 = tor ? dY * dY + dZ + dZ : dY * dY + 1.0;
    const double iden1 = rcp(den1);
    const double g1 = dX * iden1;
    const double s1 = 1.0 + dX * g1;
    const double u = rsqrt(s1);
    const double v = -dY * u * g1, w = tor ? -dZ * u * g1 : -u * g1;
    const double G0 = dX * dX + dY * dY + dZ * dZ;
    const double num = r.cX * dX + r.cY * dY + r.cZ * dZ;
    const double dot = r.cX * u + r.cY * v + r.cZ * w;
    const double iG0 = rcp(G0);
    const double av = m * num * iG0, bv = (K + L * L - 2.0 * L * m * dot) * iG0;
    const double d2 = av * av - bv, isq = rsqrt(d2), sq = d2 * isq;
    const double G = -av + sg * sq;
    // c' = m c - L uvw + G dF
    const double gG = a.cX * dX + a.cY * dY + a.cZ * dZ;
    double gX = a.cX * G, gY = a.cY * G, gZ = a.cZ * G;
    double gL = -(a.cX * u + a.cY * v + a.cZ * w);
    double gu = -L * a.cX, gv = -L * a.cY, gw = -L * a.cZ;
    a.cX *= m;
    a.cY *= m;
    a.cZ *= m;
    const double ga = -gG + sg * gG * av * isq, gb = -sg * gG * 0.5 * isq;
    const double gbn = gb * iG0;
    double gG0 = -gb * bv * iG0;
    gL += gbn * (2.0 * L - 2.0 * m * dot);
    const double gdot = -2.0 * L * m * gbn;
    a.cX += gdot * u;
    a.cY += gdot * v;
    a.cZ += gdot * w;
    gu += gdot * r.cX;
    gv += gdot * r.cY;
    gw += gdot * r.cZ;
    const double gn = ga * m * iG0;
    gG0 += -ga * av * iG0;
    a.cX += gn * dX;
    a.cY += gn * dY;
    a.cZ += gn * dZ;
    gX += gn * r.cX + 2.0 * gG0 * dX;
    gY += gn * r.cY + 2.0 * gG0 * dY;
    gZ += gn * r.cZ + 2.0 * gG0 * dZ;
    // u, v, w from the slopes
    double gg1;
    if (tor) {
        gZ += -gw * u * g1;
        gu += -gw * dZ * g1;
        gg1 = -gw * dZ * u;
    } else {
        gu += -gw * g1;
        gg1 = -gw * u;
    }
    gY += -gv * u * g1;
    gu += -gv * dY * g1;
    gg1 += -gv * dY * u;
    const double gs1 = -0.5 * gu * u * u * u;
    gX += gs1 * g1;
    gg1 += gs1 * dX;
    gX += gg1 * iden1;
    const double gden1 = -gg1 * g1 * iden1;
    gY += 2.0 * gden1 * dY;
    if (tor) gZ += 2.0 * gden1;
    slopes_rev<Sh>(s, tor, r.X, r.Y, r.Z, gX, gY, gZ, a, p);
    return gL;
}

// r: the state before the action; in: the adjoint after it.
template <class Sh = RtShape>
__device__ __forceinline__ void action_rev(const DevSurface& s, double mu, double L, const f64::Ray& r, RayA& a,
                                           SurfA& p) {
    const bool tor = Sh::cls(s) == RTB_TORIC;
    if (Sh::type(s) == RTB_MIRROR) {
        if (Sh::cls(s) == RTB_PLANE) a.cZ = -a.cZ;
        else if (Sh::cls(s) == RTB_CONIC || tor) reflect_rev<Sh>(s, tor, r, a, p);
        return;
    }
    if (Sh::type(s) == RTB_LENS) {
        if (Sh::cls(s) == RTB_PLANE) {  // a = mu cZ, G = -a + sqrt(a^2 - (mu^2 - 1)), c' = (mu cX, mu cY, mu cZ + G)
            const double av = mu * r.cZ;
            const double isq = rsqrt(av * av - (mu * mu - 1.0));
            const double gG = a.cZ;
            a.cX *= mu;
            a.cY *= mu;
            a.cZ = mu * a.cZ + mu * (-gG + gG * av * isq);
        } else if (Sh::cls(s) == RTB_CONIC || tor) {
            refract_rev<Sh>(s, tor, mu, r, a, p);
        }
        return;
    }
    if (Sh::type(s) != RTB_GRATING) return;
    const bool trans = Sh::gr_type(s) == RTB_TRANSPARENT;
    double gL = 0.0;
    if (Sh::cls(s) == RTB_PLANE) {
        // transparent: a = mu cZ, b = mu^2 - 1 + L^2 - 2 mu L cX, G = -a + sqrt(a^2 - b),
        //   c' = (mu cX - L, mu cY, mu cZ + G);
        // reflective: a = cZ, b = L^2 - 2 L cX, G = -a - sqrt(a^2 - b), c' = (cX - L, cY, cZ + G)
        const double m = trans ? mu : 1.0, K = trans ? mu * mu - 1.0 : 0.0, sg = trans ? 1.0 : -1.0;
        const double av = m * r.cZ, bv = K + L * L - 2.0 * m * L * r.cX;
        const double isq = rsqrt(av * av - bv);
        const double gG = a.cZ;
        gL = -a.cX;
        a.cX *= m;
        a.cY *= m;
        a.cZ *= m;
        const double ga = -gG + sg * gG * av * isq, gb = -sg * gG * 0.5 * isq;
        gL += gb * (2.0 * L - 2.0 * m * r.cX);
        a.cX += gb * (-2.0 * m * L);
        a.cZ += ga * m;
    } else if (Sh::cls(s) == RTB_CONIC || tor) {
        gL = diffract_curved_rev<Sh>(s, tor, trans, mu, L, r, a, p);
    }
    p.gr += gL * (-L * s.inv_gr);  // L = (order lambda / n2) / gr
}

// ---- one surface -----------------------------------------------------------------

// Surface s on one ray from its input state r0: in, the adjoint of the
// surface's output state; out, the adjoint of its input state, with the
// constants' adjoints added to p.  False if the recomputation loses the ray
// (it does not for a ray the forward traced through).
template <class Sh = RtShape>
__device__ __forceinline__ bool surface_rev(const DevSurface& s, uint32_t fixes, const double* knots,
                                            long long order, double lambda, const f64::Ray& r0, RayA& a,
                                            SurfA& p) {
    f64::Ray r1 = r0;
    f64::transform<Sh>(s, r1);
    f64::Ray r2 = r1;
    f64::normalize(r2.cX, r2.cY, r2.cZ);
    if (Sh::non_aux(s)) {
        f64::Ray r3 = r2;
        double t;
        if (!isect_fwd<Sh>(s, fixes, r3, t)) return false;
        double mu, L;
        if (!action_consts<Sh>(s, knots, order, lambda, mu, L)) return false;
        f64::Ray r4 = r3;
        if (!action_fwd<Sh>(s, mu, L, r4)) return false;
        normalize_rev(r4.cX, r4.cY, r4.cZ, a);
        action_rev<Sh>(s, mu, L, r3, a, p);
        isect_rev<Sh>(s, fixes, r2, t, a, p);
    }
    normalize_rev(r1.cX, r1.cY, r1.cZ, a);
    transform_rev(s, r0, a, p);
    return true;
}

// The adjoint of scheme parameter `ref` (a parameter of surface s) from the
// surface's constant adjoints; the chain from the parameter to the constants
// is the one make_surfd seeds.
__device__ __forceinline__ double param_adjoint(const DevSurface& s, const ad::ParamRef& ref, const SurfA& p) {
    const int i = ref.index;
    switch (ref.kind) {
        case ad::PK_CURVATURE: return p.c;
        case ad::PK_CONIC: return p.k1;
        case ad::PK_TORIC_CR: return p.cR;
        case ad::PK_POLY: {
            double v = 0.0;
#pragma unroll
            for (int j = 0; j < RTB_MAX_POLY; ++j)
                if (j == i) v = p.poly[j];
            return v;
        }
        case ad::PK_DISTANCE: return (i == 0) ? p.dist[0] : (i == 1) ? p.dist[1] : p.dist[2];
        case ad::PK_ANGLE: {  // degrees: d sinA = cosA pi/180, d cosA = -sinA pi/180
            const double gs = (i == 0) ? p.sA[0] : (i == 1) ? p.sA[1] : p.sA[2];
            const double gc = (i == 0) ? p.cA[0] : (i == 1) ? p.cA[1] : p.cA[2];
            const double sA = (i == 0) ? s.sinA[0] : (i == 1) ? s.sinA[1] : s.sinA[2];
            const double cA = (i == 0) ? s.cosA[0] : (i == 1) ? s.cosA[1] : s.cosA[2];
            return (gs * cA - gc * sA) * K_DEG2RAD;
        }
        case ad::PK_GROOVE_DENSITY: return -p.gr * s.gr_const * s.gr_const / 1000.0;  // gr = 1000 / rho
        default: return 0.0;
    }
}

}  // namespace rv
}  // namespace rtb
