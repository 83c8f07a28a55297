// rt_oracle.hpp -- CPU oracle for the ray-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU in plain FP64,
// the arithmetic of the amirych/rt CUDA engine (cuda_engine/*.cu) and of the
// host-side loops of its Beam/Surface/TabulatedFunction classes
// (common-lib/*.cpp).  It is the checker for the CUDA engine in rt_b200/:
// only tests/, __graft_entry__.smoke() and bench.py's CPU baseline may call
// it.  Nothing in the product links or executes it.
//
// Every function cites the reference file:line it follows.  Expressions keep
// the reference's operation order so that, compiled with -ffp-contract=off
// (no FMA contraction), the results are bit-identical to an IEEE FP64 device
// path compiled with --fmad=false.
//
// Parity pins: the host-side functions (Normalize, Rearrange, ApplyConstrains,
// spline evaluation, the per-surface loop) are checked against the reference's
// own host classes compiled from its sources (oracle/ref_harness.cpp,
// oracle/Makefile); the device math is checked against the reference
// cuda_engine built for sm_100a through the same harness (golden fixtures in
// tests/golden/).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstddef>
#include <cstring>
#include <vector>
#include <algorithm>

namespace rto {

// ---------------------------------------------------------------------------
// Enumerations with the reference's numbering (common-lib/surface.h:130-132,
// common-lib/surface.h:241, common-lib/beam.h:31-34).
enum SurfaceClass { Plane = 0, Conic = 1, Toric = 2, AuxClass = 3 };
enum SurfaceType { Mirror = 0, Lens = 1, Grating = 2, Stop = 3, Shade = 4, Detector = 5, AuxType = 6 };
enum SurfaceShape { Circle = 0, Rectangle = 1 };
enum GratingType { Reflective = 0, Transparent = 1 };

// Status codes; 0..4 are RT_engine_error (common-lib/rt_engine_errors.h:4-5).
enum Status { OK = 0, INIT_FAILED = 1, BAD_ALLOC = 2, FAILED = 3, BAD_VALUE = 4,
              NO_INTERSECTIONS = 5, NO_GOOD_RAYS = 6, OUT_OF_RANGE = 7 };

// Constants (common-lib/num_defs.h:20,31; cuda_engine/rt_cuda_engine_beam.cu:41;
// cuda_engine/rt_cuda_engine_ccd.cu:19; cuda_engine/rt_cuda_engine_surface.cu:667-668).
constexpr double RTO_PI = 3.14159265359;   // RT_PI
// `x *= deg2rad` expands to `x *= RTO_PI/180.0`: the factor is folded first.
constexpr double DEG2RAD_FACTOR = RTO_PI / 180.0;
constexpr double PI2 = 6.28318531;
constexpr double HC = 1.98644560233e-12;
constexpr double ITER_EPS = 1.0e-7;
constexpr size_t ITER_MAX = 100000;
constexpr int RTO_MAX_POLY = 10;   // MAX_POLY_COEFFS, common-lib/surface.h:14

// ---------------------------------------------------------------------------
// Flags for reference behaviours that are bugs.  The
// default (0) reproduces the reference; each bit switches one to the
// mathematically correct form.
enum QuirkFix : uint32_t {
    FIX_NONE = 0,
    FIX_TORIC_SIGN = 1u << 0,      // iter_toric uses 1+k1c^2Y^2 (surface.cu:350)
    FIX_TORIC_STEP = 1u << 1,      // iter_toric divides by Fzn-Fxn == 0 (surface.cu:390)
    FIX_ASPHERE_ROOT = 1u << 2,    // iterative asphere reports the point before the last Newton update (surface.cu:288-290)
};

// ---------------------------------------------------------------------------
// Surface constants as copy_surf_params() stages them
// (cuda_engine/rt_cuda_engine_surface.cu:108-148).
// T is the scalar type of the per-ray arithmetic: double for the oracle
// proper; other types (the operation counter of flop_count.hpp) take the
// same statements.
template <class T>
struct SurfConstT {
    T c = 0, k1 = 1, cR = 0;
    size_t n_poly = 0;
    T poly[RTO_MAX_POLY] = {};
    SurfConstT() = default;
    template <class U>
    explicit SurfConstT(const SurfConstT<U>& o) : c(o.c), k1(o.k1), cR(o.cR), n_poly(o.n_poly) {
        for (int i = 0; i < RTO_MAX_POLY; ++i) poly[i] = o.poly[i];
    }
};
using SurfConst = SurfConstT<double>;

inline Status make_surf_const(int cls, const double* params, SurfConst& s) {
    s.c = params[0];
    s.k1 = params[1] + 1;
    double nn = params[2];
    if (!(nn >= 0) || nn > RTO_MAX_POLY) return BAD_VALUE;
    s.n_poly = (size_t)nn;
    for (size_t i = 0; i < s.n_poly; ++i) s.poly[i] = params[3 + i];
    s.cR = (cls == Toric) ? params[3 + s.n_poly] : 0.0;
    return OK;
}

// ---------------------------------------------------------------------------
// Ray state (one ray of the SoA beam, common-lib/beam.h:96-99).
template <class T>
struct RayT {
    T X, Y, Z, cX, cY, cZ;
};
using Ray = RayT<double>;

using std::fabs;
using std::sqrt;

// ===========================================================================
// Surface derivatives
// ===========================================================================

// conic_derivs (cuda_engine/rt_cuda_engine_surface.cu:45-61)
template <class T>
inline void conic_derivs(const SurfConstT<T>& s, T X, T Y, T& dFdX, T& dFdY) {
    T r2 = X * X + Y * Y;
    T E = s.c / sqrt(1.0 - s.k1 * s.c * s.c * r2);
    T sum = 0.0, rr = 1.0;
    for (size_t i = 1; i <= s.n_poly; ++i, rr *= r2) sum += i * s.poly[i - 1] * rr;
    E += 2.0 * sum;
    dFdX = -E * X;
    dFdY = -E * Y;
}

// toric_derivs (cuda_engine/rt_cuda_engine_surface.cu:65-94)
template <class T>
inline void toric_derivs(const SurfConstT<T>& s, T X, T Y, T Z,
                         T& dFdX, T& dFdY, T& dFdZ) {
    T Y2 = Y * Y;
    T Fy = s.c * Y2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * Y2));
    T sum = 0.0, rr = Y2;
    for (size_t i = 0; i < s.n_poly; ++i, rr *= Y2) sum += s.poly[i] * rr;
    Fy += sum;
    T dFy = s.c * Y / sqrt(1.0 - s.k1 * s.c * s.c * Y2);
    sum = 0.0; rr = 1.0;
    for (size_t i = 1; i <= s.n_poly; ++i, rr *= Y2) sum += i * s.poly[i - 1] * rr;
    dFy += 2.0 * sum;
    dFdX = -s.cR * X;
    dFdY = (s.cR * Fy - 1.0) * dFy;
    dFdZ = 1.0 - s.cR * Z;
}

// ===========================================================================
// Intersection (each returns false when the ray is lost)
// ===========================================================================

// plane_intersection (surface.cu:154-178)
template <class T>
inline bool plane_intersection(RayT<T>& r) {
    T s0 = -r.Z / r.cZ;
    if (s0 < 0.0) return false;
    r.X += r.cX * s0;
    r.Y += r.cY * s0;
    r.Z = 0.0;
    return true;
}

// paraboloid_intersection (surface.cu:183-213): linear root, A ignored.
template <class T>
inline bool paraboloid_intersection(const SurfConstT<T>& s, RayT<T>& r) {
    T B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ / s.c);
    T C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z / s.c;
    T t = -C / B;
    if (t < 0.0) return false;
    r.X += t * r.cX;
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

// conic_intersection (surface.cu:216-253): root chosen by sign(c), no t>=0 check.
template <class T>
inline bool conic_intersection(const SurfConstT<T>& s, RayT<T>& r) {
    T A = s.k1 * r.cZ * r.cZ + r.cX * r.cX + r.cY * r.cY;
    T B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ / s.c);
    T C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z / s.c;
    T D = B * B - 4.0 * A * C;
    if (D < 0.0) return false;
    T t;
    if (s.c > 0) t = (-B - sqrt(D)) / 2.0 / A;
    else         t = (-B + sqrt(D)) / 2.0 / A;
    r.X += t * r.cX;
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

// iterative_conic_intersection (surface.cu:257-333).  Newton on the even
// asphere sag from the Z=0 plane point; the reported point is the last
// evaluated one (s1), written even when the ray is lost inside the loop --
// with `fix_root`, the point of the last update (s2) once converged.
// The iteration counter is reset per ray (the reference keeps it per thread
// across its grid-stride loop, which only matters after ~1e5 iterations).
template <class T>
inline bool iterative_conic_intersection(const SurfConstT<T>& s, bool fix_root, RayT<T>& r) {
    T s0 = -r.Z / r.cZ;
    if (!(s0 >= 0)) return false;
    T s1, s2 = 0.0, Xi = 0, Yi = 0, Zi = 0;
    size_t Niter = 0;
    bool good = true;
    do {
        s1 = s2;
        Xi = r.X + (s1 + s0) * r.cX;
        Yi = r.Y + (s1 + s0) * r.cY;
        Zi = s1 * r.cZ;
        T r2 = Xi * Xi + Yi * Yi;
        T F = Zi - s.c * r2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * r2));
        T sum = 0.0, rr = r2;
        for (size_t i = 0; i < s.n_poly; ++i, rr *= r2) sum += s.poly[i] * rr;
        F -= sum;
        T E = s.c / sqrt(1.0 - s.k1 * s.c * s.c * r2);
        sum = 0.0; rr = 1.0;
        for (size_t i = 1; i <= s.n_poly; ++i, rr *= r2) sum += i * s.poly[i - 1] * rr;
        E += 2.0 * sum;
        T dF = -E * Xi * r.cX - E * Yi * r.cY + r.cZ;
        if (fabs(dF) < ITER_EPS) { good = false; break; }
        s2 = s1 - F / dF;
        ++Niter;
    } while ((fabs(s2 - s1) >= ITER_EPS) && (Niter <= ITER_MAX));
    if (fix_root && good && Niter <= ITER_MAX) {  // the point of the last update
        Xi = r.X + (s2 + s0) * r.cX;
        Yi = r.Y + (s2 + s0) * r.cY;
        Zi = s2 * r.cZ;
    }
    r.X = Xi; r.Y = Yi; r.Z = Zi;
    if (Niter > ITER_MAX) good = false;
    return good;
}

// iterative_poly_intersection (surface.cu:497-561): c == 0 with a polynomial;
// requires s0 > 0 and uses (-X-Y)*sum in the derivative, as the reference.
template <class T>
inline bool iterative_poly_intersection(const SurfConstT<T>& s, bool fix_root, RayT<T>& r) {
    T s0 = -r.Z / r.cZ;
    if (!(s0 > 0)) return false;
    T s1, s2 = 0.0, Xi = 0, Yi = 0, Zi = 0;
    size_t Niter = 0;
    bool good = true;
    do {
        s1 = s2;
        Xi = r.X + (s1 + s0) * r.cX;
        Yi = r.Y + (s1 + s0) * r.cY;
        Zi = s1 * r.cZ;
        T r2 = Xi * Xi + Yi * Yi;
        T F = 0.0, rr = r2;
        for (size_t i = 0; i < s.n_poly; ++i, rr *= r2) F += s.poly[i] * rr;
        F = Zi - F;
        T dF = 0.0;
        rr = 1.0;
        for (size_t i = 1; i <= s.n_poly; ++i, rr *= r2) dF += i * s.poly[i - 1] * rr;
        dF = -Xi * dF - Yi * dF + 1.0;
        if (fabs(dF) < ITER_EPS) { good = false; break; }
        s2 = s1 - F / dF;
        ++Niter;
    } while ((fabs(s2 - s1) >= ITER_EPS) && (Niter <= ITER_MAX));
    if (fix_root && good && Niter <= ITER_MAX) {  // the point of the last update
        Xi = r.X + (s2 + s0) * r.cX;
        Yi = r.Y + (s2 + s0) * r.cY;
        Zi = s2 * r.cZ;
    }
    r.X = Xi; r.Y = Yi; r.Z = Zi;
    if (Niter > ITER_MAX) good = false;
    return good;
}

// toric_func (surface.cu:338-356); `fix_sign` selects 1-k1c^2Y^2.
template <class T>
inline T toric_func(const SurfConstT<T>& s, bool fix_sign, T t, const RayT<T>& r) {
    T X = r.X + t * r.cX;
    T Y = r.Y + t * r.cY;
    T Z = r.Z + t * r.cZ;
    T Y2 = Y * Y;
    T FY = fix_sign ? s.c * Y2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * Y2))
                         : s.c * Y2 / (1.0 + sqrt(1.0 + s.k1 * s.c * s.c * Y2));
    return Z - FY - 0.5 * s.cR * (X * X + Z * Z - FY * FY);
}

// iter_toric (surface.cu:359-410): Steffensen iteration; a ray that runs out
// of iterations is not flagged, as in the reference.  `fix_step` stops the
// iteration where the reference's step divides by Fzn-Fxn == 0.
template <class T>
inline bool iter_toric(const SurfConstT<T>& s, bool fix_sign, bool fix_step, RayT<T>& r) {
    T sn1 = -r.Z / r.cZ;
    if (!(sn1 >= 0)) return false;
    size_t Niter = 0;
    T Fyn = 0.0, sn;
    do {
        sn = sn1;
        T Fxn = toric_func(s, fix_sign, sn, r);
        if (fabs(Fyn - Fxn) <= ITER_EPS) break;
        T zn = sn + Fxn;
        T Fzn = toric_func(s, fix_sign, zn, r);
        if (fix_step && Fzn - Fxn == 0.0) { sn1 = sn; break; }
        sn1 = sn - Fxn * Fxn / (Fzn - Fxn);
        Fyn = Fxn;
        ++Niter;
    } while ((fabs(sn1 - sn) >= ITER_EPS) && (Niter <= ITER_MAX));
    r.X += sn1 * r.cX;
    r.Y += sn1 * r.cY;
    r.Z += sn1 * r.cZ;
    return true;
}

// Kind of intersection a surface uses, as engine_intersection_cycle dispatches
// (surface.cu:593-636).
enum IsectKind { IS_NONE = 0, IS_PLANE, IS_PARABOLOID, IS_CONIC, IS_ITER_POLY, IS_ITER_CONIC, IS_TORIC };

inline IsectKind intersection_kind(int cls, const double* params) {
    switch (cls) {
        case Plane: return IS_PLANE;
        case Conic: {
            size_t NN = (size_t)params[2];
            if (NN == 0) {
                if (params[0] == 0) return IS_PLANE;
                if (params[1] == -1) return IS_PARABOLOID;
                return IS_CONIC;
            }
            if (params[0] == 0) return IS_ITER_POLY;
            return IS_ITER_CONIC;
        }
        case Toric: return IS_TORIC;
        default: return IS_NONE;
    }
}

template <class T>
inline bool intersect(IsectKind kind, const SurfConstT<T>& s, uint32_t fixes, RayT<T>& r) {
    switch (kind) {
        case IS_PLANE: return plane_intersection(r);
        case IS_PARABOLOID: return paraboloid_intersection(s, r);
        case IS_CONIC: return conic_intersection(s, r);
        case IS_ITER_POLY: return iterative_poly_intersection(s, (fixes & FIX_ASPHERE_ROOT) != 0, r);
        case IS_ITER_CONIC: return iterative_conic_intersection(s, (fixes & FIX_ASPHERE_ROOT) != 0, r);
        case IS_TORIC: return iter_toric(s, (fixes & FIX_TORIC_SIGN) != 0, (fixes & FIX_TORIC_STEP) != 0, r);
        default: return true;
    }
}

// ===========================================================================
// Reflection (surface.cu:771-827)
// ===========================================================================
template <class T>
inline void reflect(int cls, const SurfConstT<T>& s, RayT<T>& r) {
    switch (cls) {
        case Plane: r.cZ = -r.cZ; return;
        case Conic: {
            T dFdX, dFdY;
            conic_derivs(s, r.X, r.Y, dFdX, dFdY);
            T a2 = 2.0 * (r.cX * dFdX + r.cY * dFdY + r.cZ) / (dFdX * dFdX + dFdY * dFdY + 1.0);
            r.cX -= a2 * dFdX;
            r.cY -= a2 * dFdY;
            r.cZ -= a2;
            return;
        }
        case Toric: {
            T dFdX, dFdY, dFdZ;
            toric_derivs(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
            T a2 = 2.0 * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) /
                        (dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ);
            r.cX -= a2 * dFdX;
            r.cY -= a2 * dFdY;
            r.cZ -= a2 * dFdZ;
            return;
        }
        default: return;
    }
}

// ===========================================================================
// Refraction (surface.cu:956-1066); mu = n1(lambda)/n2(lambda).
// ===========================================================================
template <class T>
inline bool refract(int cls, const SurfConstT<T>& s, T mu, RayT<T>& r) {
    switch (cls) {
        case Plane: {
            T a = mu * r.cZ;
            T b = mu * mu - 1.0;
            T a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            T G = -a + sqrt(b);
            r.cX *= mu;
            r.cY *= mu;
            r.cZ = mu * r.cZ + G;
            return true;
        }
        case Conic: {
            T dFdX, dFdY;
            conic_derivs(s, r.X, r.Y, dFdX, dFdY);
            T G = dFdX * dFdX + dFdY * dFdY + 1.0;
            T a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
            T b = (mu * mu - 1.0) / G;
            T a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            G = -a + sqrt(b);
            r.cX = mu * r.cX + G * dFdX;
            r.cY = mu * r.cY + G * dFdY;
            r.cZ = mu * r.cZ + G;
            return true;
        }
        case Toric: {
            T dFdX, dFdY, dFdZ;
            toric_derivs(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
            T G = dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
            T a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
            T b = (mu * mu - 1.0) / G;
            T a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            G = -a + sqrt(b);
            r.cX = mu * r.cX + G * dFdX;
            r.cY = mu * r.cY + G * dFdY;
            r.cZ = mu * r.cZ + G * dFdZ;
            return true;
        }
        default: return true;
    }
}

// ===========================================================================
// Diffraction (surface.cu:1247-1520); L = m*lambda/n2(lambda)/d.
// ===========================================================================
template <class T>
inline bool diffract(int cls, int gr_type, const SurfConstT<T>& s, T mu, T L, RayT<T>& r) {
    if (gr_type == Transparent) {
        switch (cls) {
            case Plane: {  // plane_diffr_trans_kernel (surface.cu:1247-1282)
                T a = mu * r.cZ;
                T b = mu * mu - 1.0 + L * L - 2.0 * mu * L * r.cX;
                T a2 = a * a;
                if (b > a2) return false;
                b = a2 - b;
                T G = -a + sqrt(b);
                r.cX = mu * r.cX - L;
                r.cY *= mu;
                r.cZ = mu * r.cZ + G;
                return true;
            }
            case Conic: {  // conic_diffr_trans_kernel (surface.cu:1320-1368)
                T dFdX, dFdY;
                conic_derivs(s, r.X, r.Y, dFdX, dFdY);
                T G = dFdX / (dFdY * dFdY + 1.0);
                T u = 1.0 / sqrt(1.0 + dFdX * G);
                T v = -dFdY * u * G;
                T w = -u * G;
                G = dFdX * dFdX + dFdY * dFdY + 1.0;
                T a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
                T b = (mu * mu - 1.0 + L * L - 2.0 * L * mu * (r.cX * u + r.cY * v + r.cZ * w)) / G;
                T a2 = a * a;
                if (b > a2) return false;
                b = a2 - b;
                G = -a + sqrt(b);
                r.cX = mu * r.cX - L * u + G * dFdX;
                r.cY = mu * r.cY - L * v + G * dFdY;
                r.cZ = mu * r.cZ - L * w + G;
                return true;
            }
            case Toric: {  // toric_diffr_trans_kernel (surface.cu:1423-1470)
                T dFdX, dFdY, dFdZ;
                toric_derivs(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
                T G = dFdX / (dFdY * dFdY + dFdZ + dFdZ);
                T u = 1.0 / sqrt(1.0 + dFdX * G);
                T v = -dFdY * u * G;
                T w = -dFdZ * u * G;
                G = dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
                T a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
                T b = (mu * mu - 1.0 + L * L - 2.0 * L * mu * (r.cX * u + r.cY * v + r.cZ * w)) / G;
                T a2 = a * a;
                if (b > a2) return false;
                b = a2 - b;
                G = -a + sqrt(b);
                r.cX = mu * r.cX - L * u + G * dFdX;
                r.cY = mu * r.cY - L * v + G * dFdY;
                r.cZ = mu * r.cZ - L * w + G * dFdZ;
                return true;
            }
            default: return true;
        }
    }
    switch (cls) {
        case Plane: {  // plane_diffr_refl_kernel (surface.cu:1284-1318)
            T a = r.cZ;
            T b = L * L - 2.0 * L * r.cX;
            T a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            T G = -a - sqrt(b);
            r.cX -= L;
            r.cZ += G;
            return true;
        }
        case Conic: {  // conic_diffr_refl_kernel (surface.cu:1370-1421)
            T dFdX, dFdY;
            conic_derivs(s, r.X, r.Y, dFdX, dFdY);
            T G = dFdX / (dFdY * dFdY + 1.0);
            T u = 1.0 / sqrt(1.0 + dFdX * G);
            T v = -dFdY * u * G;
            T w = -u * G;
            G = dFdX * dFdX + dFdY * dFdY + 1.0;
            T a = (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
            T b = (L * L - 2.0 * L * (r.cX * u + r.cY * v + r.cZ * w)) / G;
            T a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            G = -a - sqrt(b);
            r.cX = r.cX - L * u + G * dFdX;
            r.cY = r.cY - L * v + G * dFdY;
            r.cZ = r.cZ - L * w + G;
            return true;
        }
        case Toric: {  // toric_diffr_refl_kernel (surface.cu:1472-1520)
            T dFdX, dFdY, dFdZ;
            toric_derivs(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
            T G = dFdX / (dFdY * dFdY + dFdZ + dFdZ);
            T u = 1.0 / sqrt(1.0 + dFdX * G);
            T v = -dFdY * u * G;
            T w = -dFdZ * u * G;
            G = dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
            T a = (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
            T b = (L * L - 2.0 * L * (r.cX * u + r.cY * v + r.cZ * w)) / G;
            T a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            G = -a - sqrt(b);
            r.cX += -L * u + G * dFdX;
            r.cY += -L * v + G * dFdY;
            r.cZ += -L * w + G * dFdZ;
            return true;
        }
        default: return true;
    }
}

// ===========================================================================
// Beam host loops
// ===========================================================================

// Beam::Normalize body (common-lib/beam.cpp:541-569)
template <class T>
inline void normalize(T& cX, T& cY, T& cZ) {
    T acX = fabs(cX), acY = fabs(cY), acZ = fabs(cZ);
    T norm;
    if (acX >= acY) {
        if (acX >= acZ) norm = acX * sqrt(1.0 + acY * acY / acX / acX + acZ * acZ / acX / acX);
        else norm = acZ * sqrt(1.0 + acX * acX / acZ / acZ + acY * acY / acZ / acZ);
    } else {
        if (acY >= acZ) norm = acY * sqrt(1.0 + acX * acX / acY / acY + acZ * acZ / acY / acY);
        else norm = acZ * sqrt(1.0 + acX * acX / acZ / acZ + acY * acY / acZ / acZ);
    }
    cX /= norm;
    cY /= norm;
    cZ /= norm;
}

// Aperture test of Surface::ApplyConstrains (common-lib/surface.cpp:264-321)
// and Shade::ApplyConstrains (common-lib/surface.cpp:652-699); true = ray
// survives.  `shade` selects the inverted test.
template <class T>
inline bool aperture_pass(bool shade, int shape, const double size[2], const double center[2],
                          T X, T Y) {
    T xr = X - center[0];
    T yr = Y - center[1];
    if (!shade) {
        if (shape == Circle) {
            const double R2 = size[0] * size[0];  // once per surface in the reference
            T ray_R2 = xr * xr + yr * yr;
            return !(ray_R2 > R2);
        }
        return !((X < (T(center[0]) - T(size[0]) / 2.0)) || (X > (T(center[0]) + T(size[0]) / 2.0)) ||
                 (Y < (T(center[1]) - T(size[1]) / 2.0)) || (Y > (T(center[1]) + T(size[1]) / 2.0)));
    }
    if (shape == Circle) {
        const double R2 = size[0] * size[0];
        T ray_R2 = xr * xr + yr * yr;
        return !(ray_R2 <= R2);
    }
    return !((xr >= -T(size[0]) / 2.0) && (xr <= T(size[0]) / 2.0) &&
             (yr >= -T(size[1]) / 2.0) && (yr <= T(size[1]) / 2.0));
}

// Beam::Rearrange (common-lib/beam.cpp:574-598): two-pointer partition of the
// good prefix [0,n_good).  `swap(i, j)` exchanges rays i and j in every array;
// returns the new number of good rays.
template <class SwapFn>
inline size_t rearrange(char* flag, size_t n_good, SwapFn swap) {
    if (n_good == 0) return 0;
    size_t start = 0;
    long long end = (long long)n_good - 1;
    size_t i = 0;
    size_t ng = n_good;
    while ((long long)start <= end) {
        while ((long long)start <= end && flag[start] == 1) { ++start; ++i; }
        while ((long long)start <= end && flag[end] == 0) { --end; --ng; }
        if ((long long)start < end) {
            flag[start] = 1;
            flag[end] = 0;
            swap(i, ng - 1);
        }
    }
    return ng;
}

// ===========================================================================
// Transform (cuda_engine/rt_cuda_engine_beam.cu:320-350,416-579)
// ===========================================================================

// Host-side angle handling: the surface keeps radians set from degrees
// (surface.cpp:201), returns degrees (surface.cpp:227) and Beam::Transform
// converts back to radians (beam.cpp:609-611).
inline double scheme_angle_rad(double deg) {
    double rad = deg * DEG2RAD_FACTOR;      // SetAngles
    double back = rad / DEG2RAD_FACTOR;     // GetAngles
    return back * DEG2RAD_FACTOR;           // Beam::Transform
}

struct TransformConst {
    double dist[3];
    bool translate;
    bool rot[3];
    double sinA[3], cosA[3];
};

// `angles` are radians as passed to beam_transform.
inline TransformConst make_transform(const double angles[3], const double dist[3]) {
    TransformConst t;
    for (int i = 0; i < 3; ++i) t.dist[i] = dist[i];
    t.translate = (dist[2] != 0.0) || (dist[0] != 0.0) || (dist[1] != 0.0);
    for (int i = 0; i < 3; ++i) {
        t.rot[i] = angles[i] != 0;
        t.sinA[i] = t.rot[i] ? std::sin(angles[i]) : 0.0;
        t.cosA[i] = t.rot[i] ? std::cos(angles[i]) : 1.0;
    }
    return t;
}

// rotation_kernel body (beam.cu:333-350)
template <class T>
inline void rotate_pair(double sA, double cA, T& v1, T& v2, T& w1, T& w2) {
    T e = v1 * cA - v2 * sA;
    v2 = v1 * sA + v2 * cA;
    v1 = e;
    e = w1 * cA - w2 * sA;
    w2 = w1 * sA + w2 * cA;
    w1 = e;
}

// Translation then rotations about Y, X, Z (beam.cu:437-518).
template <class T>
inline void transform(const TransformConst& t, RayT<T>& r) {
    if (t.translate) {
        r.X -= t.dist[0];
        r.Y -= t.dist[1];
        r.Z -= t.dist[2];
    }
    if (t.rot[0]) rotate_pair(t.sinA[0], t.cosA[0], r.X, r.Z, r.cX, r.cZ);
    if (t.rot[1]) rotate_pair(t.sinA[1], t.cosA[1], r.Y, r.Z, r.cY, r.cZ);
    if (t.rot[2]) rotate_pair(t.sinA[2], t.cosA[2], r.X, r.Y, r.cX, r.cY);
}

// ===========================================================================
// Tabulated function (common-lib/tabulated_function.cpp)
// ===========================================================================
struct Table {
    bool single = true;
    std::vector<double> x, y, y2;
};

// Natural cubic spline second derivatives, the sequential Numerical Recipes
// algorithm that rt_cuda_engine_spline.cu:43-145 parallelises (and races on).
inline void spline_init(size_t N, const double* x, const double* y, double* y2) {
    std::vector<double> u(N, 0.0);
    y2[0] = 0.0;
    y2[N - 1] = 0.0;
    u[0] = 0.0;
    for (size_t i = 1; i + 1 < N; ++i) {
        double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
        double p = sig * y2[i - 1] + 2.0;
        y2[i] = (sig - 1.0) / p;
        u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
        u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
    }
    for (size_t k = N - 2; k > 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
}

// TabulatedFunction::operator[] (tabulated_function.cpp:173-204).  Returns
// false where the reference throws (OutOfRange, BadArgument).
template <class T>
inline bool table_eval(size_t n, const double* x, const double* y, const double* y2, T xval, T& out) {
    if (n == 0) return false;
    if (n == 1) { out = y[0]; return true; }
    if ((xval < x[0]) || (xval > x[n - 1])) return false;
    size_t il = 0, ir = n, i;
    while ((ir - il) > 1) {
        i = (il + ir) >> 1;
        if (x[i] == xval) { out = y[i]; return true; }
        if (x[i] > xval) ir = i; else il = i;
    }
    T h = T(x[ir]) - x[il];
    if (h == 0.0) return false;
    T a = (x[ir] - xval) / h;
    T b = (xval - x[il]) / h;
    out = a * y[il] + b * y[ir] + ((a * a * a - a) * y2[il] + (b * b * b - b) * y2[ir]) * (h * h) / 6.0;
    return true;
}

// ===========================================================================
// CCD (cuda_engine/rt_cuda_engine_ccd.cu)
// ===========================================================================

// __double2uint_rz as the device converts: truncation toward zero,
// saturating (negative -> 0, >= 2^32 -> 0xFFFFFFFF), NaN -> 0x80000000
// (measured on B200: tests/test_gpu_parity.py).
inline uint32_t double2uint_rz(double v) {
    if (v != v) return 0x80000000u;
    if (!(v > 0.0)) return 0u;
    if (v >= 4294967296.0) return 0xFFFFFFFFu;
    return (uint32_t)v;                   // C++ conversion truncates toward zero
}

// ccd_coordinates_kernel (ccd.cu:30-45)
inline void ccd_coords(double X, double Y, double xsize, double ysize, double xpix, double ypix,
                       uint32_t& ix, uint32_t& iy) {
    ix = double2uint_rz((X + xsize / 2.0) / xpix);
    iy = double2uint_rz((Y + ysize / 2.0) / ypix);
}

// ===========================================================================
// Philox4x32-10 counter-based generator (Salmon et al., "Parallel random
// numbers: as easy as 1, 2, 3", SC'11) and the seeded synthetic beam.
// ===========================================================================
struct U4 { uint32_t v[4]; };

inline U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)M0 * ctr.v[0];
        uint64_t p1 = (uint64_t)M1 * ctr.v[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        U4 n;
        n.v[0] = hi1 ^ ctr.v[1] ^ k0;
        n.v[1] = lo1;
        n.v[2] = hi0 ^ ctr.v[3] ^ k1;
        n.v[3] = lo0;
        ctr = n;
        k0 += W0;
        k1 += W1;
    }
    return ctr;
}

// Uniform double in (0,1] from 64 random bits: ((b >> 11) + 1) * 2^-53.
inline double u01_from_bits(uint32_t hi, uint32_t lo) {
    uint64_t b = ((uint64_t)hi << 32) | lo;
    return (double)((b >> 11) + 1) * (1.0 / 9007199254740992.0);
}

// Two uniforms for ray `ray` of stream `stream` under `seed`.
inline void ray_uniforms(uint64_t seed, uint64_t stream, uint64_t ray, double& u1, double& u2) {
    U4 c;
    c.v[0] = (uint32_t)ray;
    c.v[1] = (uint32_t)(ray >> 32);
    c.v[2] = (uint32_t)stream;
    c.v[3] = (uint32_t)(stream >> 32);
    U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    u1 = u01_from_bits(r.v[0], r.v[1]);
    u2 = u01_from_bits(r.v[2], r.v[3]);
}

// sin and cos of x for the beam generator, evaluated identically on CPU and
// GPU: Cody-Waite reduction by pi/2 with a three-part constant (Cody & Waite,
// "Software Manual for the Elementary Functions", 1980) and Taylor series on
// [-pi/4, pi/4] to degree 19/20 evaluated by Horner's rule.  Valid for
// |x| < 1e5; the generator only calls it on [0, 2*pi).
inline void beam_sincos(double x, double& s, double& c) {
    const double INV_PIO2 = 0.6366197723675814;            // 2/pi
    const double P1 = 1.5707963267341256e+00;              // pi/2, 33 bits
    const double P2 = 6.077100506303966e-11;               // next 33 bits
    const double P3 = 2.0222662487959506e-21;              // remainder
    double k = std::nearbyint(x * INV_PIO2);
    double r = ((x - k * P1) - k * P2) - k * P3;
    double r2 = r * r;
    // sin(r) = r * (1 - r2/3! + r2^2/5! - ...), cos(r) = 1 - r2/2! + ...
    double ps = 1.0 / 121645100408832000.0;                 // 1/19!
    ps = ps * (-r2) + 1.0 / 355687428096000.0;              // 1/17!
    ps = ps * (-r2) + 1.0 / 1307674368000.0;                // 1/15!
    ps = ps * (-r2) + 1.0 / 6227020800.0;                   // 1/13!
    ps = ps * (-r2) + 1.0 / 39916800.0;                     // 1/11!
    ps = ps * (-r2) + 1.0 / 362880.0;                       // 1/9!
    ps = ps * (-r2) + 1.0 / 5040.0;                         // 1/7!
    ps = ps * (-r2) + 1.0 / 120.0;                          // 1/5!
    ps = ps * (-r2) + 1.0 / 6.0;                            // 1/3!
    ps = ps * (-r2) + 1.0;
    double sr = r * ps;
    double pc = 1.0 / 2432902008176640000.0;                // 1/20!
    pc = pc * (-r2) + 1.0 / 6402373705728000.0;             // 1/18!
    pc = pc * (-r2) + 1.0 / 20922789888000.0;               // 1/16!
    pc = pc * (-r2) + 1.0 / 87178291200.0;                  // 1/14!
    pc = pc * (-r2) + 1.0 / 479001600.0;                    // 1/12!
    pc = pc * (-r2) + 1.0 / 3628800.0;                      // 1/10!
    pc = pc * (-r2) + 1.0 / 40320.0;                        // 1/8!
    pc = pc * (-r2) + 1.0 / 720.0;                          // 1/6!
    pc = pc * (-r2) + 1.0 / 24.0;                           // 1/4!
    pc = pc * (-r2) + 1.0 / 2.0;                            // 1/2!
    double cr = 1.0 - r2 * pc;
    long q = (long)k & 3;
    switch (q) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}

// Uniform disk position (random_circle_kernel, beam.cu:126-152) from the
// seeded uniforms.  params = [N, R_in, R_out], center = [x, y, z].
inline void disk_position(const double params[3], const double center[3], double u1, double u2,
                          double& X, double& Y, double& Z) {
    double phi = PI2 * u2;
    Z = center[2];
    double R = (params[2] - params[1]) * std::sqrt(u1) + params[1];
    double sp, cp;
    beam_sincos(phi, sp, cp);
    X = R * cp + center[0];
    Y = R * sp + center[1];
}

// uniform_range_beam_kernel (beam.cu:701-710) with the step of
// uniform_range_beam (beam.cu:726).
inline double uniform_lambda(const double range[2], size_t n_lambda, size_t j) {
    double d_l = (range[1] - range[0]) / (n_lambda - 1);
    return range[0] + j * d_l;
}

// ===========================================================================
// Grating blaze efficiency (the throughput curves of Scheme::ComputeQE)
// ===========================================================================

// __double2ll_rz for the finite, in-range values the order bounds take:
// truncation toward zero.
inline long long double2ll_rz(double v) { return (long long)v; }

// I1_func_Tarasov (rt_cuda_engine_surface.cu:1988-2019) in double: blaze
// angle c, incidence k1 (alpha), grating constant eps, relative rule length
// rule_size; the small-argument branch is the reference's series for
// sin(u)/u.
inline double i1_tarasov(double c, double k1, double eps, double rule_size, double lambda, double beta) {
    double I1 = RTO_PI * eps * rule_size / lambda * std::cos(beta) / std::cos(c - beta) *
                (std::sin(c - k1) + std::sin(c - beta));
    double term = std::cos(beta) * std::cos(c - k1) / std::cos(c - beta);
    if (std::fabs(I1) < RTO_PI / 2.0) {
        I1 *= I1;
        I1 = (0.00761 * I1 - 0.16605) * I1 + 1;
    } else {
        I1 = std::sin(I1) / (I1);
    }
    I1 *= term;
    I1 *= I1;
    return I1;
}

// grating_energy_distr_kernel (rt_cuda_engine_surface.cu:2098-2153) for one
// wavelength: I1 in `order` over the sum of I1 over every order from
// trunc(eps/lambda*(sin(alpha)-1)*cos(gamma)) to trunc(eps/lambda*(sin(alpha)+1)*cos(gamma)).
inline double grating_energy(double l, long order, double blaze, double alpha, double gamma, double eps,
                             double rule_size) {
    double sin_alpha = std::sin(alpha);
    double cos_gamma = std::cos(gamma);
    long order_min = (long)double2ll_rz(eps / l * (sin_alpha - 1) * cos_gamma);
    long order_max = (long)double2ll_rz(eps / l * (sin_alpha + 1) * cos_gamma);
    double norm = 0.0;
    for (long m = order_min; m <= order_max; ++m) {
        double beta = std::asin(m * l / eps / cos_gamma - sin_alpha);
        norm += i1_tarasov(blaze, alpha, eps, rule_size, l, beta);
    }
    double beta = std::asin(order * l / (eps * cos_gamma) - sin_alpha);
    double I1 = i1_tarasov(blaze, alpha, eps, rule_size, l, beta);
    return I1 / norm;
}

}  // namespace rto
