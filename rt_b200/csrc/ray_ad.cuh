// ray_ad.cuh -- the plain FP64 engine's per-ray arithmetic on dual numbers.
//
// Each function restates the function of the same name in ray_fp64.cuh (and
// through it the reference kernel it cites) statement for statement, with the
// ray state and the differentiable surface constants as Dual<W>: the values
// are the plain engine's bits, the tangents their derivatives.  Branches
// (lost-ray tests, normalisation order) follow the values.
//
// Root iterations (asphere Newton, toric Steffensen) run on the values exactly
// as the plain engine runs them; the tangent of the root comes from the
// implicit-function theorem at the point the iteration returns:
// dt = -(dF/dinputs) / (dF/dt), with F the surface function along the ray.
#pragma once

#include "dual.cuh"
#include "ray_fp64.cuh"
#include "shape.cuh"

namespace rtb {
namespace ad {

// Which field of a DevSurface a scheme parameter moves (rtb_param.kind).
enum ParamKind : int32_t {
    PK_CURVATURE = RTB_PARAM_CURVATURE,
    PK_CONIC = RTB_PARAM_CONIC,
    PK_POLY = RTB_PARAM_POLY,
    PK_TORIC_CR = RTB_PARAM_TORIC_CR,
    PK_DISTANCE = RTB_PARAM_DISTANCE,
    PK_ANGLE = RTB_PARAM_ANGLE,
    PK_GROOVE_DENSITY = RTB_PARAM_GROOVE_DENSITY
};

struct ParamRef {
    int32_t surface, kind, index, pad;
};

template <int W>
struct RayD {
    Dual<W> X, Y, Z, cX, cY, cZ;
};

// The differentiable constants of one surface.
template <int W>
struct SurfD {
    Dual<W> c, k1, cR, gr;
    Dual<W> poly[RTB_MAX_POLY];
    Dual<W> dist[3], sinA[3], cosA[3];
    bool seeded_dist, seeded_angle[3];
};

// Seeds of one pass: lane l differentiates either state component
// state[l] (0..5: X Y Z cX cY cZ), or parameter param[l] (unit direction),
// or -- with `dense` set, lane 0 only -- the parameter direction dense[0..P).
template <int W>
struct Seeds {
    int state[W];
    int param[W];
    const double* dense;
};

template <int W>
__device__ __forceinline__ void seed_field(Dual<W>& f, int lane, double w) {
    f.d[lane] += w;
}

template <int W>
__device__ void make_surfd(const DevSurface& s, int k, const ParamRef* map, int n_params, const Seeds<W>& sd,
                           SurfD<W>& o) {
    o.c = cst<W>(s.c);
    o.k1 = cst<W>(s.k1);
    o.cR = cst<W>(s.cR);
    o.gr = cst<W>(s.gr_const);
    for (int i = 0; i < RTB_MAX_POLY; ++i) o.poly[i] = cst<W>(s.poly[i]);
    for (int i = 0; i < 3; ++i) {
        o.dist[i] = cst<W>(s.dist[i]);
        o.sinA[i] = cst<W>(s.sinA[i]);
        o.cosA[i] = cst<W>(s.cosA[i]);
        o.seeded_angle[i] = false;
    }
    o.seeded_dist = false;
    for (int j = 0; j < n_params; ++j) {
        const ParamRef p = map[j];
        if (p.surface != k) continue;
        for (int l = 0; l < W; ++l) {
            double w = 0.0;
            if (sd.dense) w = (l == 0) ? sd.dense[j] : 0.0;
            else w = (sd.param[l] == j) ? 1.0 : 0.0;
            if (w == 0.0) continue;
            switch (p.kind) {
                case PK_CURVATURE: seed_field(o.c, l, w); break;
                case PK_CONIC: seed_field(o.k1, l, w); break;
                case PK_POLY: seed_field(o.poly[p.index], l, w); break;
                case PK_TORIC_CR: seed_field(o.cR, l, w); break;
                case PK_DISTANCE:
                    seed_field(o.dist[p.index], l, w);
                    o.seeded_dist = true;
                    break;
                case PK_ANGLE:  // degrees; d(rad)/d(deg) = pi/180 of the reference's round trip
                    seed_field(o.sinA[p.index], l, w * s.cosA[p.index] * K_DEG2RAD);
                    seed_field(o.cosA[p.index], l, -w * s.sinA[p.index] * K_DEG2RAD);
                    o.seeded_angle[p.index] = true;
                    break;
                case PK_GROOVE_DENSITY:  // gr_const = 1000 / rho (lines/mm -> microns)
                    seed_field(o.gr, l, -w * s.gr_const * s.gr_const / 1000.0);
                    break;
                default: break;
            }
        }
    }
}

// The seeded component is chosen with selects, not by indexing: a run-time
// index into the ray's fields would keep the whole ray in local memory.
// State seeds: lane l differentiates component sd.state[l] (0..5), or the
// cosines along t1 (6) or t2 (7).
template <int W>
__device__ __forceinline__ void load_state(const double st[6], const Seeds<W>& sd, RayD<W>& r,
                                           const double* t1 = nullptr, const double* t2 = nullptr) {
    r.X = cst<W>(st[0]);
    r.Y = cst<W>(st[1]);
    r.Z = cst<W>(st[2]);
    r.cX = cst<W>(st[3]);
    r.cY = cst<W>(st[4]);
    r.cZ = cst<W>(st[5]);
    if (sd.dense) return;
#pragma unroll
    for (int l = 0; l < W; ++l) {
        const int c = sd.state[l];
        r.X.d[l] = (c == 0) ? 1.0 : 0.0;
        r.Y.d[l] = (c == 1) ? 1.0 : 0.0;
        r.Z.d[l] = (c == 2) ? 1.0 : 0.0;
        r.cX.d[l] = (c == 3) ? 1.0 : (c == 6 && t1) ? t1[0] : (c == 7 && t2) ? t2[0] : 0.0;
        r.cY.d[l] = (c == 4) ? 1.0 : (c == 6 && t1) ? t1[1] : (c == 7 && t2) ? t2[1] : 0.0;
        r.cZ.d[l] = (c == 5) ? 1.0 : (c == 6 && t1) ? t1[2] : (c == 7 && t2) ? t2[2] : 0.0;
    }
}

// ---- surface derivatives --------------------------------------------------

template <int W>
__device__ __forceinline__ void conic_derivs(const SurfD<W>& s, int n_poly, const Dual<W>& X, const Dual<W>& Y,
                                             Dual<W>& dFdX, Dual<W>& dFdY) {
    Dual<W> r2 = X * X + Y * Y;
    Dual<W> E = s.c / sqrt(1.0 - s.k1 * s.c * s.c * r2);
    Dual<W> sum = cst<W>(0.0), rr = cst<W>(1.0);
    for (int i = 1; i <= n_poly; ++i, rr *= r2) sum += (double)i * s.poly[i - 1] * rr;
    E += 2.0 * sum;
    dFdX = -E * X;
    dFdY = -E * Y;
}

template <int W>
__device__ __forceinline__ void toric_derivs(const SurfD<W>& s, int n_poly, const Dual<W>& X, const Dual<W>& Y,
                                             const Dual<W>& Z, Dual<W>& dFdX, Dual<W>& dFdY, Dual<W>& dFdZ) {
    Dual<W> Y2 = Y * Y;
    Dual<W> Fy = s.c * Y2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * Y2));
    Dual<W> sum = cst<W>(0.0), rr = Y2;
    for (int i = 0; i < n_poly; ++i, rr *= Y2) sum += s.poly[i] * rr;
    Fy += sum;
    Dual<W> dFy = s.c * Y / sqrt(1.0 - s.k1 * s.c * s.c * Y2);
    sum = cst<W>(0.0);
    rr = cst<W>(1.0);
    for (int i = 1; i <= n_poly; ++i, rr *= Y2) sum += (double)i * s.poly[i - 1] * rr;
    dFy += 2.0 * sum;
    dFdX = -s.cR * X;
    dFdY = (s.cR * Fy - 1.0) * dFy;
    dFdZ = 1.0 - s.cR * Z;
}

// ---- transform and normalisation --------------------------------------------

template <int W>
__device__ __forceinline__ void rotate_pair(const Dual<W>& sA, const Dual<W>& cA, Dual<W>& v1, Dual<W>& v2,
                                            Dual<W>& w1, Dual<W>& w2) {
    Dual<W> e = v1 * cA - v2 * sA;
    v2 = v1 * sA + v2 * cA;
    v1 = e;
    e = w1 * cA - w2 * sA;
    w2 = w1 * sA + w2 * cA;
    w1 = e;
}

// beam_transform (rt_cuda_engine_beam.cu:416-579).  A rotation or translation
// the plain engine skips (zero angle or distance) is applied when its
// parameter is seeded: the values are unchanged, the tangent is not.
template <int W>
__device__ __forceinline__ void transform(const DevSurface& s, const SurfD<W>& sd, RayD<W>& r) {
    if (s.translate || sd.seeded_dist) {
        r.X -= sd.dist[0];
        r.Y -= sd.dist[1];
        r.Z -= sd.dist[2];
    }
    if ((s.rot_mask & 1) || sd.seeded_angle[0]) rotate_pair(sd.sinA[0], sd.cosA[0], r.X, r.Z, r.cX, r.cZ);
    if ((s.rot_mask & 2) || sd.seeded_angle[1]) rotate_pair(sd.sinA[1], sd.cosA[1], r.Y, r.Z, r.cY, r.cZ);
    if ((s.rot_mask & 4) || sd.seeded_angle[2]) rotate_pair(sd.sinA[2], sd.cosA[2], r.X, r.Y, r.cX, r.cY);
}

// Beam::Normalize body (beam.cpp:541-569)
template <int W>
__device__ __forceinline__ void normalize(Dual<W>& cX, Dual<W>& cY, Dual<W>& cZ) {
    Dual<W> acX = fabs(cX), acY = fabs(cY), acZ = fabs(cZ);
    Dual<W> norm;
    if (acX.v >= acY.v) {
        if (acX.v >= acZ.v) norm = acX * sqrt(1.0 + acY * acY / acX / acX + acZ * acZ / acX / acX);
        else norm = acZ * sqrt(1.0 + acX * acX / acZ / acZ + acY * acY / acZ / acZ);
    } else {
        if (acY.v >= acZ.v) norm = acY * sqrt(1.0 + acX * acX / acY / acY + acZ * acZ / acY / acY);
        else norm = acZ * sqrt(1.0 + acX * acX / acZ / acZ + acY * acY / acZ / acZ);
    }
    cX /= norm;
    cY /= norm;
    cZ /= norm;
}

// ---- intersections -----------------------------------------------------------

template <int W>
__device__ __forceinline__ bool plane_isect(RayD<W>& r) {
    Dual<W> s0 = -r.Z / r.cZ;
    if (s0.v < 0.0) return false;
    r.X += r.cX * s0;
    r.Y += r.cY * s0;
    r.Z = cst<W>(0.0);
    return true;
}

template <int W>
__device__ __forceinline__ bool paraboloid_isect(const SurfD<W>& s, RayD<W>& r) {
    Dual<W> B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ / s.c);
    Dual<W> C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z / s.c;
    Dual<W> t = -C / B;
    if (t.v < 0.0) return false;
    r.X += t * r.cX;
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

template <int W>
__device__ __forceinline__ bool conic_isect(const SurfD<W>& s, RayD<W>& r) {
    Dual<W> A = s.k1 * r.cZ * r.cZ + r.cX * r.cX + r.cY * r.cY;
    Dual<W> B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ / s.c);
    Dual<W> C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z / s.c;
    Dual<W> D = B * B - 4.0 * A * C;
    if (D.v < 0.0) return false;
    Dual<W> t;
    if (s.c.v > 0) t = (-B - sqrt(D)) / 2.0 / A;
    else t = (-B + sqrt(D)) / 2.0 / A;
    r.X += t * r.cX;
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

// Even asphere (iterative_conic_intersection / iterative_poly_intersection):
// the iteration on the values, as f64::iter_*_isect runs it, returning the
// offset s1 of the point it reports (measured from the plane point s0).
__device__ __forceinline__ bool asphere_values(const DevSurface& s, const f64::Ray& r, bool poly_only, bool fix_root,
                                               double& s1_out) {
    double s0 = -r.Z / r.cZ;
    if (poly_only ? !(s0 > 0) : !(s0 >= 0)) return false;
    double s1, s2 = 0.0;
    unsigned niter = 0;
    bool good = true;
    f64::CycleSkip cyc;
    do {
        s1 = s2;
        double Xi = r.X + (s1 + s0) * r.cX;
        double Yi = r.Y + (s1 + s0) * r.cY;
        double Zi = s1 * r.cZ;
        double r2 = Xi * Xi + Yi * Yi;
        double F, dF;
        if (!poly_only) {
            F = Zi - s.c * r2 / (1.0 + ::sqrt(1.0 - s.k1 * s.c * s.c * r2));
            double sum = 0.0, rr = r2;
            for (int i = 0; i < s.n_poly; ++i, rr *= r2) sum += s.poly[i] * rr;
            F -= sum;
            double E = s.c / ::sqrt(1.0 - s.k1 * s.c * s.c * r2);
            sum = 0.0;
            rr = 1.0;
            for (int i = 1; i <= s.n_poly; ++i, rr *= r2) sum += (double)i * s.poly[i - 1] * rr;
            E += 2.0 * sum;
            dF = -E * Xi * r.cX - E * Yi * r.cY + r.cZ;
        } else {
            F = 0.0;
            double rr = r2;
            for (int i = 0; i < s.n_poly; ++i, rr *= r2) F += s.poly[i] * rr;
            F = Zi - F;
            dF = 0.0;
            rr = 1.0;
            for (int i = 1; i <= s.n_poly; ++i, rr *= r2) dF += (double)i * s.poly[i - 1] * rr;
            dF = -Xi * dF - Yi * dF + 1.0;
        }
        if (::fabs(dF) < K_ITER_EPS) {
            good = false;
            break;
        }
        s2 = s1 - F / dF;
        ++niter;
        cyc.step(s2, 0.0, niter);
    } while ((::fabs(s2 - s1) >= K_ITER_EPS) && (niter <= K_ITER_MAX));
    if (niter > K_ITER_MAX) good = false;
    s1_out = (fix_root && good) ? s2 : s1;
    return good;
}

// Surface function of the even asphere at a point (conic sag + polynomial).
template <int W>
__device__ __forceinline__ Dual<W> asphere_F(const SurfD<W>& s, int n_poly, bool poly_only, const Dual<W>& X,
                                             const Dual<W>& Y, const Dual<W>& Z) {
    Dual<W> r2 = X * X + Y * Y;
    Dual<W> sag = cst<W>(0.0);
    if (!poly_only) sag = s.c * r2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * r2));
    Dual<W> rr = r2;
    for (int i = 0; i < n_poly; ++i, rr *= r2) sag += s.poly[i] * rr;
    return Z - sag;
}

template <int W>
__device__ __forceinline__ bool asphere_isect(const DevSurface& ds, const SurfD<W>& s, bool poly_only, uint32_t fixes,
                                              RayD<W>& r) {
    f64::Ray rv{r.X.v, r.Y.v, r.Z.v, r.cX.v, r.cY.v, r.cZ.v};
    double s1;
    if (!asphere_values(ds, rv, poly_only, (fixes & RTB_FIX_ASPHERE_ROOT) != 0, s1)) return false;  // lost
    Dual<W> s0 = -r.Z / r.cZ;
    // the reported point P = ray(s0 + s1); its parameter t moves with the
    // inputs as -F_inputs / F_t (F evaluated at P with t held fixed)
    Dual<W> tfix = cst<W>(s1 + s0.v);
    Dual<W> X = r.X + tfix * r.cX, Y = r.Y + tfix * r.cY, Z = r.Z + tfix * r.cZ;
    Dual<W> F = asphere_F(s, ds.n_poly, poly_only, X, Y, Z);
    // dF/dt along the ray at P (exact derivative of the surface function)
    const double r2 = X.v * X.v + Y.v * Y.v;
    double E = 0.0;
    if (!poly_only) E = ds.c / ::sqrt(1.0 - ds.k1 * ds.c * ds.c * r2);
    double sum = 0.0, rr = 1.0;
    for (int i = 1; i <= ds.n_poly; ++i, rr *= r2) sum += (double)i * ds.poly[i - 1] * rr;
    E += 2.0 * sum;
    const double Ft = rv.cZ - E * (X.v * rv.cX + Y.v * rv.cY);
    Dual<W> tsum;
    tsum.v = s1 + s0.v;
    const double iFt = tangent_rcp(Ft);
#pragma unroll
    for (int l = 0; l < W; ++l) tsum.d[l] = -F.d[l] * iFt;
    Dual<W> Xi = r.X + tsum * r.cX;
    Dual<W> Yi = r.Y + tsum * r.cY;
    Dual<W> Zi = r.Z + tsum * r.cZ;
    Zi.v = s1 * r.cZ.v;  // the reference reports Zi = s1 * cZ (surface.cu:288-290)
    r.X = Xi;
    r.Y = Yi;
    r.Z = Zi;
    return true;
}

// Toric surface function along the ray (toric_func, surface.cu:338-356).
template <int W>
__device__ __forceinline__ Dual<W> toric_F(const SurfD<W>& s, bool fix_sign, const Dual<W>& X, const Dual<W>& Y,
                                           const Dual<W>& Z) {
    Dual<W> Y2 = Y * Y;
    Dual<W> FY = fix_sign ? s.c * Y2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * Y2))
                          : s.c * Y2 / (1.0 + sqrt(1.0 + s.k1 * s.c * s.c * Y2));
    return Z - FY - 0.5 * s.cR * (X * X + Z * Z - FY * FY);
}

// The toric iteration on the values, as f64::toric_isect runs it; sn1 is the
// ray parameter of the point it reports.
__device__ __forceinline__ bool toric_values(const DevSurface& s, uint32_t fixes, const f64::Ray& r, double& sn1_out) {
    const bool fix_sign = (fixes & RTB_FIX_TORIC_SIGN) != 0;
    const bool fix_step = (fixes & RTB_FIX_TORIC_STEP) != 0;
    double sn1 = -r.Z / r.cZ;
    if (!(sn1 >= 0)) return false;
    unsigned niter = 0;
    double Fyn = 0.0, sn;
    f64::CycleSkip cyc;
    do {
        sn = sn1;
        double Fxn = f64::toric_func(s, fix_sign, sn, r);
        if (::fabs(Fyn - Fxn) <= K_ITER_EPS) break;
        double zn = sn + Fxn;
        double Fzn = f64::toric_func(s, fix_sign, zn, r);
        if (fix_step && Fzn - Fxn == 0.0) {
            sn1 = sn;
            break;
        }
        sn1 = sn - Fxn * Fxn / (Fzn - Fxn);
        Fyn = Fxn;
        ++niter;
        cyc.step(sn1, Fyn, niter);
    } while ((::fabs(sn1 - sn) >= K_ITER_EPS) && (niter <= K_ITER_MAX));
    sn1_out = sn1;
    return true;
}

template <int W>
__device__ __forceinline__ bool toric_isect(const DevSurface& ds, const SurfD<W>& s, uint32_t fixes, RayD<W>& r) {
    const bool fix_sign = (fixes & RTB_FIX_TORIC_SIGN) != 0;
    f64::Ray rv{r.X.v, r.Y.v, r.Z.v, r.cX.v, r.cY.v, r.cZ.v};
    double sn1;
    if (!toric_values(ds, fixes, rv, sn1)) return false;
    Dual<W> tfix = cst<W>(sn1);
    Dual<W> X = r.X + tfix * r.cX, Y = r.Y + tfix * r.cY, Z = r.Z + tfix * r.cZ;
    Dual<W> F = toric_F(s, fix_sign, X, Y, Z);
    // dF/dt = cZ - FY' cY - cR (X cX + Z cZ - FY FY' cY), FY' = c Y / sqrt(1 -+ k1 c^2 Y^2)
    const double sg = fix_sign ? -1.0 : 1.0;
    const double Yv = Y.v, Y2 = Yv * Yv;
    const double q = ::sqrt(1.0 + sg * ds.k1 * ds.c * ds.c * Y2);
    const double FY = ds.c * Y2 / (1.0 + q), dFY = ds.c * Yv / q;
    const double Ft = rv.cZ - dFY * rv.cY - ds.cR * (X.v * rv.cX + Z.v * rv.cZ - FY * dFY * rv.cY);
    Dual<W> t;
    t.v = sn1;
    const double iFt = tangent_rcp(Ft);
#pragma unroll
    for (int l = 0; l < W; ++l) t.d[l] = -F.d[l] * iFt;
    r.X += t * r.cX;  // values: X + sn1 * cX, as the plain engine
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

template <int W, class Sh = RtShape>
__device__ __forceinline__ bool intersect(const DevSurface& ds, const SurfD<W>& s, uint32_t fixes, RayD<W>& r) {
    switch (Sh::kind(ds)) {
        case IS_PLANE: return plane_isect(r);
        case IS_PARABOLOID: return paraboloid_isect(s, r);
        case IS_CONIC: return conic_isect(s, r);
        case IS_ITER_POLY: return asphere_isect(ds, s, true, fixes, r);
        case IS_ITER_CONIC: return asphere_isect(ds, s, false, fixes, r);
        case IS_TORIC: return toric_isect(ds, s, fixes, r);
        default: return true;
    }
}

// ---- actions -------------------------------------------------------------------

template <int W, class Sh = RtShape>
__device__ __forceinline__ void reflect(const DevSurface& ds, const SurfD<W>& s, RayD<W>& r) {
    if (Sh::cls(ds) == RTB_PLANE) {
        r.cZ = -r.cZ;
    } else if (Sh::cls(ds) == RTB_CONIC) {
        Dual<W> dFdX, dFdY;
        conic_derivs(s, Sh::n_poly(ds), r.X, r.Y, dFdX, dFdY);
        Dual<W> a2 = 2.0 * (r.cX * dFdX + r.cY * dFdY + r.cZ) / (dFdX * dFdX + dFdY * dFdY + 1.0);
        r.cX -= a2 * dFdX;
        r.cY -= a2 * dFdY;
        r.cZ -= a2;
    } else if (Sh::cls(ds) == RTB_TORIC) {
        Dual<W> dFdX, dFdY, dFdZ;
        toric_derivs(s, Sh::n_poly(ds), r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
        Dual<W> a2 = 2.0 * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / (dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ);
        r.cX -= a2 * dFdX;
        r.cY -= a2 * dFdY;
        r.cZ -= a2 * dFdZ;
    }
}

template <int W, class Sh = RtShape>
__device__ __forceinline__ bool refract(const DevSurface& ds, const SurfD<W>& s, double mu, RayD<W>& r) {
    if (Sh::cls(ds) == RTB_PLANE) {
        Dual<W> a = mu * r.cZ;
        double b = mu * mu - 1.0;
        Dual<W> a2 = a * a;
        if (b > a2.v) return false;
        Dual<W> bb = a2 - b;
        Dual<W> G = -a + sqrt(bb);
        r.cX *= mu;
        r.cY *= mu;
        r.cZ = mu * r.cZ + G;
        return true;
    }
    Dual<W> dFdX, dFdY, dFdZ = cst<W>(1.0);
    if (Sh::cls(ds) == RTB_CONIC) conic_derivs(s, Sh::n_poly(ds), r.X, r.Y, dFdX, dFdY);
    else toric_derivs(s, Sh::n_poly(ds), r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
    Dual<W> G = (Sh::cls(ds) == RTB_CONIC) ? dFdX * dFdX + dFdY * dFdY + 1.0 : dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
    Dual<W> a = (Sh::cls(ds) == RTB_CONIC) ? mu * (r.cX * dFdX + r.cY * dFdY + r.cZ) / G
                                      : mu * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
    Dual<W> b = (mu * mu - 1.0) / G;
    Dual<W> a2 = a * a;
    if (b.v > a2.v) return false;
    b = a2 - b;
    G = -a + sqrt(b);
    r.cX = mu * r.cX + G * dFdX;
    r.cY = mu * r.cY + G * dFdY;
    r.cZ = (Sh::cls(ds) == RTB_CONIC) ? mu * r.cZ + G : mu * r.cZ + G * dFdZ;
    return true;
}

template <int W, class Sh = RtShape>
__device__ __forceinline__ bool diffract(const DevSurface& ds, const SurfD<W>& s, double mu, const Dual<W>& L,
                                         RayD<W>& r) {
    if (Sh::gr_type(ds) == RTB_TRANSPARENT) {
        if (Sh::cls(ds) == RTB_PLANE) {
            Dual<W> a = mu * r.cZ;
            Dual<W> b = mu * mu - 1.0 + L * L - 2.0 * mu * L * r.cX;
            Dual<W> a2 = a * a;
            if (b.v > a2.v) return false;
            b = a2 - b;
            Dual<W> G = -a + sqrt(b);
            r.cX = mu * r.cX - L;
            r.cY *= mu;
            r.cZ = mu * r.cZ + G;
            return true;
        }
        Dual<W> dFdX, dFdY, dFdZ = cst<W>(1.0);
        const bool tor = Sh::cls(ds) == RTB_TORIC;
        if (tor) toric_derivs(s, Sh::n_poly(ds), r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
        else conic_derivs(s, Sh::n_poly(ds), r.X, r.Y, dFdX, dFdY);
        Dual<W> G = tor ? dFdX / (dFdY * dFdY + dFdZ + dFdZ) : dFdX / (dFdY * dFdY + 1.0);
        Dual<W> u = 1.0 / sqrt(1.0 + dFdX * G);
        Dual<W> v = -dFdY * u * G;
        Dual<W> w = tor ? -dFdZ * u * G : -u * G;
        G = tor ? dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ : dFdX * dFdX + dFdY * dFdY + 1.0;
        Dual<W> a = tor ? mu * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G : mu * (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
        Dual<W> b = (mu * mu - 1.0 + L * L - 2.0 * L * mu * (r.cX * u + r.cY * v + r.cZ * w)) / G;
        Dual<W> a2 = a * a;
        if (b.v > a2.v) return false;
        b = a2 - b;
        G = -a + sqrt(b);
        r.cX = mu * r.cX - L * u + G * dFdX;
        r.cY = mu * r.cY - L * v + G * dFdY;
        r.cZ = tor ? mu * r.cZ - L * w + G * dFdZ : mu * r.cZ - L * w + G;
        return true;
    }
    if (Sh::cls(ds) == RTB_PLANE) {
        Dual<W> a = r.cZ;
        Dual<W> b = L * L - 2.0 * L * r.cX;
        Dual<W> a2 = a * a;
        if (b.v > a2.v) return false;
        b = a2 - b;
        Dual<W> G = -a - sqrt(b);
        r.cX -= L;
        r.cZ += G;
        return true;
    }
    Dual<W> dFdX, dFdY, dFdZ = cst<W>(1.0);
    const bool tor = Sh::cls(ds) == RTB_TORIC;
    if (tor) toric_derivs(s, Sh::n_poly(ds), r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
    else conic_derivs(s, Sh::n_poly(ds), r.X, r.Y, dFdX, dFdY);
    Dual<W> G = tor ? dFdX / (dFdY * dFdY + dFdZ + dFdZ) : dFdX / (dFdY * dFdY + 1.0);
    Dual<W> u = 1.0 / sqrt(1.0 + dFdX * G);
    Dual<W> v = -dFdY * u * G;
    Dual<W> w = tor ? -dFdZ * u * G : -u * G;
    G = tor ? dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ : dFdX * dFdX + dFdY * dFdY + 1.0;
    Dual<W> a = tor ? (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G : (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
    Dual<W> b = (L * L - 2.0 * L * (r.cX * u + r.cY * v + r.cZ * w)) / G;
    Dual<W> a2 = a * a;
    if (b.v > a2.v) return false;
    b = a2 - b;
    G = -a - sqrt(b);
    if (tor) {
        r.cX += -L * u + G * dFdX;
        r.cY += -L * v + G * dFdY;
        r.cZ += -L * w + G * dFdZ;
    } else {
        r.cX = r.cX - L * u + G * dFdX;
        r.cY = r.cY - L * v + G * dFdY;
        r.cZ = r.cZ - L * w + G;
    }
    return true;
}

// Mirror/Lens/Grating ::Action (f64::action); refractive indices depend on
// the wavelength only, the grating constant on its groove density.
template <int W, class Sh = RtShape>
__device__ __forceinline__ int action(const DevSurface& ds, const SurfD<W>& s, const double* knots, long long order,
                                      double lambda, RayD<W>& r) {
    if (Sh::type(ds) == RTB_MIRROR) {
        reflect<W, Sh>(ds, s, r);
        return f64::ACT_OK;
    }
    if (Sh::type(ds) == RTB_LENS) {
        double a, b;
        if (!f64::table_eval(knots + ds.n1_off, ds.n1_n, lambda, a) ||
            !f64::table_eval(knots + ds.n2_off, ds.n2_n, lambda, b))
            return f64::ACT_RANGE;
        double mu = a;
        mu /= b;
        return refract<W, Sh>(ds, s, mu, r) ? f64::ACT_OK : f64::ACT_LOST;
    }
    if (Sh::type(ds) == RTB_GRATING) {
        double n2v, mu = 0.0;
        if (!f64::table_eval(knots + ds.n2_off, ds.n2_n, lambda, n2v)) return f64::ACT_RANGE;
        if (Sh::gr_type(ds) == RTB_TRANSPARENT) {
            double n1v;
            if (!f64::table_eval(knots + ds.n1_off, ds.n1_n, lambda, n1v)) return f64::ACT_RANGE;
            mu = n1v;
            mu /= n2v;
        }
        Dual<W> L = cst<W>((double)order * lambda / n2v) / s.gr;
        return diffract<W, Sh>(ds, s, mu, L, r) ? f64::ACT_OK : f64::ACT_LOST;
    }
    return f64::ACT_OK;
}

// One surface on one ray, as the fused FP64 kernel runs it: transform,
// normalise, and for a non-Aux surface intersection, aperture, action and
// normalise.  True if the ray survives.
template <int W, class Sh = RtShape>
__device__ __forceinline__ bool surface_step(const DevSurface& ds, const SurfD<W>& s, uint32_t fixes,
                                             const double* knots, long long order, double lambda, RayD<W>& r) {
    transform(ds, s, r);
    normalize(r.cX, r.cY, r.cZ);
    if (!Sh::non_aux(ds)) return true;
    if (!intersect<W, Sh>(ds, s, fixes, r)) return false;
    if (!f64::aperture_pass(Sh::type(ds) == RTB_SHADE, Sh::shape(ds), ds.size, ds.center, r.X.v, r.Y.v)) return false;
    if (action<W, Sh>(ds, s, knots, order, lambda, r) != f64::ACT_OK) return false;
    normalize(r.cX, r.cY, r.cZ);
    return true;
}

}  // namespace ad
}  // namespace rtb
