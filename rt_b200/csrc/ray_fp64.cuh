// ray_fp64.cuh -- per-ray FP64 arithmetic of the plain engine.
//
// Each function restates one kernel body of the reference CUDA engine
// (cuda_engine/rt_cuda_engine_*.cu, cited per function) or one host loop body
// of its classes, keeping the reference's operation order.  Translation units
// that include this file are compiled with --fmad=false, so every result is
// the IEEE-rounded value of the same expression the CPU oracle evaluates:
// the plain engine is bit-identical to the oracle (NaN payloads aside).
#pragma once

#include "common.cuh"
#include "shape.cuh"

namespace rtb {
namespace f64 {

struct Ray {
    double X, Y, Z, cX, cY, cZ;
};

// The reference's root iterations stop only on convergence or after
// K_ITER_MAX steps.  A few rays never converge: their iterate falls into an
// exact cycle (on the C1 echelle's toric fold, 5 of 8.7e7 rays enter a
// 2-cycle after 5 Steffensen steps) and would hold their warp for 1e5 steps.
// Each iteration is a pure function of a small state, so once the state's
// bit pattern repeats after `lam` steps it repeats forever: the remaining
// steps up to the cap can be skipped in whole periods, and the loop then runs
// the last (< lam) steps as usual.  The result is the same bits as running
// every step.  Cycles are found with Brent's algorithm (R. P. Brent, "An
// improved Monte Carlo factorization algorithm", BIT 20, 1980), armed only
// after K_CYCLE_FROM steps so converging rays pay one compare per step.
constexpr unsigned K_CYCLE_FROM = 8;

struct CycleSkip {
    unsigned long long a = 0, b = 0;  // saved state (bit patterns)
    unsigned power = 1, lam = 0;
    bool armed = false;

    // Call after the step that brought the counter to `niter`, with the
    // state (x, y) the next step starts from; may advance `niter`.
    __device__ __forceinline__ void step(double x, double y, unsigned& niter) {
        if (niter < K_CYCLE_FROM) return;
        const unsigned long long xb = (unsigned long long)__double_as_longlong(x);
        const unsigned long long yb = (unsigned long long)__double_as_longlong(y);
        if (!armed) {
            armed = true;
            a = xb;
            b = yb;
            return;
        }
        ++lam;
        if (xb == a && yb == b) {
            const unsigned left = K_ITER_MAX + 1 - niter;  // steps until the cap ends the loop
            niter += left - left % lam;
        } else if (lam == power) {
            a = xb;
            b = yb;
            power <<= 1;
            lam = 0;
        }
    }
};

// conic_derivs (rt_cuda_engine_surface.cu:45-61)
template <class Sh = RtShape>
__device__ __forceinline__ void conic_derivs(const DevSurface& s, double X, double Y, double& dFdX, double& dFdY) {
    double r2 = X * X + Y * Y;
    double E = s.c / sqrt(1.0 - s.k1 * s.c * s.c * r2);
    double sum = 0.0, rr = 1.0;
    for (int i = 1; i <= Sh::n_poly(s); ++i, rr *= r2) sum += (double)i * s.poly[i - 1] * rr;
    E += 2.0 * sum;
    dFdX = -E * X;
    dFdY = -E * Y;
}

// toric_derivs (rt_cuda_engine_surface.cu:65-94)
template <class Sh = RtShape>
__device__ __forceinline__ void toric_derivs(const DevSurface& s, double X, double Y, double Z, double& dFdX,
                                             double& dFdY, double& dFdZ) {
    double Y2 = Y * Y;
    double Fy = s.c * Y2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * Y2));
    double sum = 0.0, rr = Y2;
    for (int i = 0; i < Sh::n_poly(s); ++i, rr *= Y2) sum += s.poly[i] * rr;
    Fy += sum;
    double dFy = s.c * Y / sqrt(1.0 - s.k1 * s.c * s.c * Y2);
    sum = 0.0;
    rr = 1.0;
    for (int i = 1; i <= Sh::n_poly(s); ++i, rr *= Y2) sum += (double)i * s.poly[i - 1] * rr;
    dFy += 2.0 * sum;
    dFdX = -s.cR * X;
    dFdY = (s.cR * Fy - 1.0) * dFy;
    dFdZ = 1.0 - s.cR * Z;
}

// ---- intersections (return false when the ray is lost) -------------------

// plane_intersection (rt_cuda_engine_surface.cu:154-178)
__device__ __forceinline__ bool plane_isect(Ray& r) {
    double s0 = -r.Z / r.cZ;
    if (s0 < 0.0) return false;
    r.X += r.cX * s0;
    r.Y += r.cY * s0;
    r.Z = 0.0;
    return true;
}

// paraboloid_intersection (rt_cuda_engine_surface.cu:183-213)
__device__ __forceinline__ bool paraboloid_isect(const DevSurface& s, Ray& r) {
    double B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ / s.c);
    double C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z / s.c;
    double t = -C / B;
    if (t < 0.0) return false;
    r.X += t * r.cX;
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

// conic_intersection (rt_cuda_engine_surface.cu:216-253)
__device__ __forceinline__ bool conic_isect(const DevSurface& s, Ray& r) {
    double A = s.k1 * r.cZ * r.cZ + r.cX * r.cX + r.cY * r.cY;
    double B = 2.0 * (s.k1 * r.Z * r.cZ + r.X * r.cX + r.Y * r.cY - r.cZ / s.c);
    double C = s.k1 * r.Z * r.Z + r.X * r.X + r.Y * r.Y - 2.0 * r.Z / s.c;
    double D = B * B - 4.0 * A * C;
    if (D < 0.0) return false;
    double t;
    if (s.c > 0) t = (-B - sqrt(D)) / 2.0 / A;
    else t = (-B + sqrt(D)) / 2.0 / A;
    r.X += t * r.cX;
    r.Y += t * r.cY;
    r.Z += t * r.cZ;
    return true;
}

// iterative_conic_intersection (rt_cuda_engine_surface.cu:257-333); the
// iteration count is per ray and bounded by K_ITER_MAX.
template <class Sh = RtShape>
__device__ __forceinline__ bool iter_conic_isect(const DevSurface& s, bool fix_root, Ray& r) {
    double s0 = -r.Z / r.cZ;
    if (!(s0 >= 0)) return false;
    double s1, s2 = 0.0, Xi = 0, Yi = 0, Zi = 0;
    unsigned niter = 0;
    bool good = true;
    CycleSkip cyc;
    do {
        s1 = s2;
        Xi = r.X + (s1 + s0) * r.cX;
        Yi = r.Y + (s1 + s0) * r.cY;
        Zi = s1 * r.cZ;
        double r2 = Xi * Xi + Yi * Yi;
        double F = Zi - s.c * r2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * r2));
        double sum = 0.0, rr = r2;
        for (int i = 0; i < Sh::n_poly(s); ++i, rr *= r2) sum += s.poly[i] * rr;
        F -= sum;
        double E = s.c / sqrt(1.0 - s.k1 * s.c * s.c * r2);
        sum = 0.0;
        rr = 1.0;
        for (int i = 1; i <= Sh::n_poly(s); ++i, rr *= r2) sum += (double)i * s.poly[i - 1] * rr;
        E += 2.0 * sum;
        double dF = -E * Xi * r.cX - E * Yi * r.cY + r.cZ;
        if (fabs(dF) < K_ITER_EPS) { good = false; break; }
        s2 = s1 - F / dF;
        ++niter;
        cyc.step(s2, 0.0, niter);
    } while ((fabs(s2 - s1) >= K_ITER_EPS) && (niter <= K_ITER_MAX));
    if (fix_root && good && niter <= K_ITER_MAX) {  // RTB_FIX_ASPHERE_ROOT: the point of the last update
        Xi = r.X + (s2 + s0) * r.cX;
        Yi = r.Y + (s2 + s0) * r.cY;
        Zi = s2 * r.cZ;
    }
    r.X = Xi;
    r.Y = Yi;
    r.Z = Zi;
    if (niter > K_ITER_MAX) good = false;
    return good;
}

// iterative_poly_intersection (rt_cuda_engine_surface.cu:497-561)
template <class Sh = RtShape>
__device__ __forceinline__ bool iter_poly_isect(const DevSurface& s, bool fix_root, Ray& r) {
    double s0 = -r.Z / r.cZ;
    if (!(s0 > 0)) return false;
    double s1, s2 = 0.0, Xi = 0, Yi = 0, Zi = 0;
    unsigned niter = 0;
    bool good = true;
    CycleSkip cyc;
    do {
        s1 = s2;
        Xi = r.X + (s1 + s0) * r.cX;
        Yi = r.Y + (s1 + s0) * r.cY;
        Zi = s1 * r.cZ;
        double r2 = Xi * Xi + Yi * Yi;
        double F = 0.0, rr = r2;
        for (int i = 0; i < Sh::n_poly(s); ++i, rr *= r2) F += s.poly[i] * rr;
        F = Zi - F;
        double dF = 0.0;
        rr = 1.0;
        for (int i = 1; i <= Sh::n_poly(s); ++i, rr *= r2) dF += (double)i * s.poly[i - 1] * rr;
        dF = -Xi * dF - Yi * dF + 1.0;
        if (fabs(dF) < K_ITER_EPS) { good = false; break; }
        s2 = s1 - F / dF;
        ++niter;
        cyc.step(s2, 0.0, niter);
    } while ((fabs(s2 - s1) >= K_ITER_EPS) && (niter <= K_ITER_MAX));
    if (fix_root && good && niter <= K_ITER_MAX) {  // RTB_FIX_ASPHERE_ROOT: the point of the last update
        Xi = r.X + (s2 + s0) * r.cX;
        Yi = r.Y + (s2 + s0) * r.cY;
        Zi = s2 * r.cZ;
    }
    r.X = Xi;
    r.Y = Yi;
    r.Z = Zi;
    if (niter > K_ITER_MAX) good = false;
    return good;
}

// toric_func (rt_cuda_engine_surface.cu:338-356)
__device__ __forceinline__ double toric_func(const DevSurface& s, bool fix_sign, double t, const Ray& r) {
    double X = r.X + t * r.cX;
    double Y = r.Y + t * r.cY;
    double Z = r.Z + t * r.cZ;
    double Y2 = Y * Y;
    double FY = fix_sign ? s.c * Y2 / (1.0 + sqrt(1.0 - s.k1 * s.c * s.c * Y2))
                         : s.c * Y2 / (1.0 + sqrt(1.0 + s.k1 * s.c * s.c * Y2));
    return Z - FY - 0.5 * s.cR * (X * X + Z * Z - FY * FY);
}

// iter_toric (rt_cuda_engine_surface.cu:359-410) without its per-ray printf.
__device__ __forceinline__ bool toric_isect(const DevSurface& s, uint32_t fixes, Ray& r) {
    const bool fix_sign = (fixes & RTB_FIX_TORIC_SIGN) != 0;
    const bool fix_step = (fixes & RTB_FIX_TORIC_STEP) != 0;
    double sn1 = -r.Z / r.cZ;
    if (!(sn1 >= 0)) return false;
    unsigned niter = 0;
    double Fyn = 0.0, sn;
    CycleSkip cyc;
    do {
        sn = sn1;
        double Fxn = toric_func(s, fix_sign, sn, r);
        if (fabs(Fyn - Fxn) <= K_ITER_EPS) break;
        double zn = sn + Fxn;
        double Fzn = toric_func(s, fix_sign, zn, r);
        if (fix_step && Fzn - Fxn == 0.0) { sn1 = sn; break; }
        sn1 = sn - Fxn * Fxn / (Fzn - Fxn);
        Fyn = Fxn;
        ++niter;
        cyc.step(sn1, Fyn, niter);
    } while ((fabs(sn1 - sn) >= K_ITER_EPS) && (niter <= K_ITER_MAX));
    r.X += sn1 * r.cX;
    r.Y += sn1 * r.cY;
    r.Z += sn1 * r.cZ;
    return true;
}

template <class Sh = RtShape>
__device__ __forceinline__ bool intersect(const DevSurface& s, uint32_t fixes, Ray& r) {
    switch (Sh::kind(s)) {
        case IS_PLANE: return plane_isect(r);
        case IS_PARABOLOID: return paraboloid_isect(s, r);
        case IS_CONIC: return conic_isect(s, r);
        case IS_ITER_POLY: return iter_poly_isect<Sh>(s, (fixes & RTB_FIX_ASPHERE_ROOT) != 0, r);
        case IS_ITER_CONIC: return iter_conic_isect<Sh>(s, (fixes & RTB_FIX_ASPHERE_ROOT) != 0, r);
        case IS_TORIC: return toric_isect(s, fixes, r);
        default: return true;
    }
}

// ---- reflection (rt_cuda_engine_surface.cu:771-827) -----------------------
template <class Sh = RtShape>
__device__ __forceinline__ void reflect(const DevSurface& s, Ray& r) {
    if (Sh::cls(s) == RTB_PLANE) {
        r.cZ = -r.cZ;
    } else if (Sh::cls(s) == RTB_CONIC) {
        double dFdX, dFdY;
        conic_derivs<Sh>(s, r.X, r.Y, dFdX, dFdY);
        double a2 = 2.0 * (r.cX * dFdX + r.cY * dFdY + r.cZ) / (dFdX * dFdX + dFdY * dFdY + 1.0);
        r.cX -= a2 * dFdX;
        r.cY -= a2 * dFdY;
        r.cZ -= a2;
    } else if (Sh::cls(s) == RTB_TORIC) {
        double dFdX, dFdY, dFdZ;
        toric_derivs<Sh>(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
        double a2 = 2.0 * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / (dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ);
        r.cX -= a2 * dFdX;
        r.cY -= a2 * dFdY;
        r.cZ -= a2 * dFdZ;
    }
}

// ---- refraction (rt_cuda_engine_surface.cu:956-1066) ----------------------
template <class Sh = RtShape>
__device__ __forceinline__ bool refract(const DevSurface& s, double mu, Ray& r) {
    if (Sh::cls(s) == RTB_PLANE) {
        double a = mu * r.cZ;
        double b = mu * mu - 1.0;
        double a2 = a * a;
        if (b > a2) return false;
        b = a2 - b;
        double G = -a + sqrt(b);
        r.cX *= mu;
        r.cY *= mu;
        r.cZ = mu * r.cZ + G;
        return true;
    }
    if (Sh::cls(s) == RTB_CONIC) {
        double dFdX, dFdY;
        conic_derivs<Sh>(s, r.X, r.Y, dFdX, dFdY);
        double G = dFdX * dFdX + dFdY * dFdY + 1.0;
        double a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
        double b = (mu * mu - 1.0) / G;
        double a2 = a * a;
        if (b > a2) return false;
        b = a2 - b;
        G = -a + sqrt(b);
        r.cX = mu * r.cX + G * dFdX;
        r.cY = mu * r.cY + G * dFdY;
        r.cZ = mu * r.cZ + G;
        return true;
    }
    if (Sh::cls(s) == RTB_TORIC) {
        double dFdX, dFdY, dFdZ;
        toric_derivs<Sh>(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
        double G = dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
        double a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
        double b = (mu * mu - 1.0) / G;
        double a2 = a * a;
        if (b > a2) return false;
        b = a2 - b;
        G = -a + sqrt(b);
        r.cX = mu * r.cX + G * dFdX;
        r.cY = mu * r.cY + G * dFdY;
        r.cZ = mu * r.cZ + G * dFdZ;
        return true;
    }
    return true;
}

// ---- diffraction (rt_cuda_engine_surface.cu:1247-1520) --------------------
template <class Sh = RtShape>
__device__ __forceinline__ bool diffract(const DevSurface& s, double mu, double L, Ray& r) {
    if (Sh::gr_type(s) == RTB_TRANSPARENT) {
        if (Sh::cls(s) == RTB_PLANE) {  // plane_diffr_trans_kernel
            double a = mu * r.cZ;
            double b = mu * mu - 1.0 + L * L - 2.0 * mu * L * r.cX;
            double a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            double G = -a + sqrt(b);
            r.cX = mu * r.cX - L;
            r.cY *= mu;
            r.cZ = mu * r.cZ + G;
            return true;
        }
        if (Sh::cls(s) == RTB_CONIC) {  // conic_diffr_trans_kernel
            double dFdX, dFdY;
            conic_derivs<Sh>(s, r.X, r.Y, dFdX, dFdY);
            double G = dFdX / (dFdY * dFdY + 1.0);
            double u = 1.0 / sqrt(1.0 + dFdX * G);
            double v = -dFdY * u * G;
            double w = -u * G;
            G = dFdX * dFdX + dFdY * dFdY + 1.0;
            double a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
            double b = (mu * mu - 1.0 + L * L - 2.0 * L * mu * (r.cX * u + r.cY * v + r.cZ * w)) / G;
            double a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            G = -a + sqrt(b);
            r.cX = mu * r.cX - L * u + G * dFdX;
            r.cY = mu * r.cY - L * v + G * dFdY;
            r.cZ = mu * r.cZ - L * w + G;
            return true;
        }
        if (Sh::cls(s) == RTB_TORIC) {  // toric_diffr_trans_kernel
            double dFdX, dFdY, dFdZ;
            toric_derivs<Sh>(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
            double G = dFdX / (dFdY * dFdY + dFdZ + dFdZ);
            double u = 1.0 / sqrt(1.0 + dFdX * G);
            double v = -dFdY * u * G;
            double w = -dFdZ * u * G;
            G = dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
            double a = mu * (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
            double b = (mu * mu - 1.0 + L * L - 2.0 * L * mu * (r.cX * u + r.cY * v + r.cZ * w)) / G;
            double a2 = a * a;
            if (b > a2) return false;
            b = a2 - b;
            G = -a + sqrt(b);
            r.cX = mu * r.cX - L * u + G * dFdX;
            r.cY = mu * r.cY - L * v + G * dFdY;
            r.cZ = mu * r.cZ - L * w + G * dFdZ;
            return true;
        }
        return true;
    }
    if (Sh::cls(s) == RTB_PLANE) {  // plane_diffr_refl_kernel
        double a = r.cZ;
        double b = L * L - 2.0 * L * r.cX;
        double a2 = a * a;
        if (b > a2) return false;
        b = a2 - b;
        double G = -a - sqrt(b);
        r.cX -= L;
        r.cZ += G;
        return true;
    }
    if (Sh::cls(s) == RTB_CONIC) {  // conic_diffr_refl_kernel
        double dFdX, dFdY;
        conic_derivs<Sh>(s, r.X, r.Y, dFdX, dFdY);
        double G = dFdX / (dFdY * dFdY + 1.0);
        double u = 1.0 / sqrt(1.0 + dFdX * G);
        double v = -dFdY * u * G;
        double w = -u * G;
        G = dFdX * dFdX + dFdY * dFdY + 1.0;
        double a = (r.cX * dFdX + r.cY * dFdY + r.cZ) / G;
        double b = (L * L - 2.0 * L * (r.cX * u + r.cY * v + r.cZ * w)) / G;
        double a2 = a * a;
        if (b > a2) return false;
        b = a2 - b;
        G = -a - sqrt(b);
        r.cX = r.cX - L * u + G * dFdX;
        r.cY = r.cY - L * v + G * dFdY;
        r.cZ = r.cZ - L * w + G;
        return true;
    }
    if (Sh::cls(s) == RTB_TORIC) {  // toric_diffr_refl_kernel
        double dFdX, dFdY, dFdZ;
        toric_derivs<Sh>(s, r.X, r.Y, r.Z, dFdX, dFdY, dFdZ);
        double G = dFdX / (dFdY * dFdY + dFdZ + dFdZ);
        double u = 1.0 / sqrt(1.0 + dFdX * G);
        double v = -dFdY * u * G;
        double w = -dFdZ * u * G;
        G = dFdX * dFdX + dFdY * dFdY + dFdZ * dFdZ;
        double a = (r.cX * dFdX + r.cY * dFdY + r.cZ * dFdZ) / G;
        double b = (L * L - 2.0 * L * (r.cX * u + r.cY * v + r.cZ * w)) / G;
        double a2 = a * a;
        if (b > a2) return false;
        b = a2 - b;
        G = -a - sqrt(b);
        r.cX += -L * u + G * dFdX;
        r.cY += -L * v + G * dFdY;
        r.cZ += -L * w + G * dFdZ;
        return true;
    }
    return true;
}

// ---- host loops of Beam/Surface -------------------------------------------

// Beam::Normalize body (common-lib/beam.cpp:541-569)
__device__ __forceinline__ void normalize(double& cX, double& cY, double& cZ) {
    double acX = fabs(cX), acY = fabs(cY), acZ = fabs(cZ);
    double norm;
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

// Normalize a lost ray `count` times, stopping at the fixed point.
__device__ __forceinline__ void renormalize(Ray& r, int count) {
    for (int i = 0; i < count; ++i) {
        double a = r.cX, b = r.cY, c = r.cZ;
        normalize(a, b, c);
        if (a == r.cX && b == r.cY && c == r.cZ) break;
        r.cX = a;
        r.cY = b;
        r.cZ = c;
    }
}

// Surface::ApplyConstrains / Shade::ApplyConstrains (surface.cpp:264-321,652-699)
__device__ __forceinline__ bool aperture_pass(bool shade, int shape, const double* size, const double* center,
                                              double X, double Y) {
    double xr = X - center[0];
    double yr = Y - center[1];
    if (!shade) {
        if (shape == RTB_CIRCLE) {
            double R2 = size[0] * size[0];
            return !(xr * xr + yr * yr > R2);
        }
        return !((X < (center[0] - size[0] / 2.0)) || (X > (center[0] + size[0] / 2.0)) ||
                 (Y < (center[1] - size[1] / 2.0)) || (Y > (center[1] + size[1] / 2.0)));
    }
    if (shape == RTB_CIRCLE) {
        double R2 = size[0] * size[0];
        return !(xr * xr + yr * yr <= R2);
    }
    return !((xr >= -size[0] / 2.0) && (xr <= size[0] / 2.0) && (yr >= -size[1] / 2.0) && (yr <= size[1] / 2.0));
}

// rotation_kernel body (rt_cuda_engine_beam.cu:333-350)
__device__ __forceinline__ void rotate_pair(double sA, double cA, double& v1, double& v2, double& w1, double& w2) {
    double e = v1 * cA - v2 * sA;
    v2 = v1 * sA + v2 * cA;
    v1 = e;
    e = w1 * cA - w2 * sA;
    w2 = w1 * sA + w2 * cA;
    w1 = e;
}

// beam_transform: translation then rotations about y, x, z (rt_cuda_engine_beam.cu:416-579)
template <class Sh = RtShape>
__device__ __forceinline__ void transform(const DevSurface& s, Ray& r) {
    if (Sh::translate(s)) {
        r.X -= s.dist[0];
        r.Y -= s.dist[1];
        r.Z -= s.dist[2];
    }
    if (Sh::rot_mask(s) & 1) rotate_pair(s.sinA[0], s.cosA[0], r.X, r.Z, r.cX, r.cZ);
    if (Sh::rot_mask(s) & 2) rotate_pair(s.sinA[1], s.cosA[1], r.Y, r.Z, r.cY, r.cZ);
    if (Sh::rot_mask(s) & 4) rotate_pair(s.sinA[2], s.cosA[2], r.X, r.Y, r.cX, r.cY);
}

// TabulatedFunction::operator[] (tabulated_function.cpp:173-204); knots at
// tab[0..n) = x, tab[n..2n) = y, tab[2n..3n) = y2; n == 1 is a single value
// stored at tab[1].  Returns false where the reference throws.
__device__ __forceinline__ bool table_eval(const double* tab, int n, double xval, double& out) {
    if (n == 1) {
        out = tab[1];
        return true;
    }
    const double* x = tab;
    const double* y = tab + n;
    const double* y2 = tab + 2 * n;
    if ((xval < x[0]) || (xval > x[n - 1])) return false;
    int il = 0, ir = n;
    while ((ir - il) > 1) {
        int i = (il + ir) >> 1;
        if (x[i] == xval) {
            out = y[i];
            return true;
        }
        if (x[i] > xval) ir = i;
        else il = i;
    }
    double h = x[ir] - x[il];
    if (h == 0.0) return false;
    double a = (x[ir] - xval) / h;
    double b = (xval - x[il]) / h;
    out = a * y[il] + b * y[ir] + ((a * a * a - a) * y2[il] + (b * b * b - b) * y2[ir]) * (h * h) / 6.0;
    return true;
}

// Result of the action of a surface on one ray.
enum ActionResult { ACT_OK = 0, ACT_LOST = 1, ACT_RANGE = 2 };

// Mirror/Lens/Grating ::Action on one ray (surface.cpp:385-396,453-472,563-585)
// with n(lambda) evaluated on the device (the reference evaluates it on the
// host per ray, surface.cu:1094-1097,1565-1569,1608-1610).
template <class Sh = RtShape>
__device__ __forceinline__ int action(const DevSurface& s, const double* knots, long long order, double lambda,
                                      Ray& r) {
    if (Sh::type(s) == RTB_MIRROR) {
        reflect<Sh>(s, r);
        return ACT_OK;
    }
    if (Sh::type(s) == RTB_LENS) {
        double a, b;
        if (!table_eval(knots + s.n1_off, s.n1_n, lambda, a) || !table_eval(knots + s.n2_off, s.n2_n, lambda, b))
            return ACT_RANGE;
        double mu = a;
        mu /= b;
        return refract<Sh>(s, mu, r) ? ACT_OK : ACT_LOST;
    }
    if (Sh::type(s) == RTB_GRATING) {
        double n2v, mu = 0.0;
        if (!table_eval(knots + s.n2_off, s.n2_n, lambda, n2v)) return ACT_RANGE;
        if (Sh::gr_type(s) == RTB_TRANSPARENT) {
            double n1v;
            if (!table_eval(knots + s.n1_off, s.n1_n, lambda, n1v)) return ACT_RANGE;
            mu = n1v;
            mu /= n2v;
        }
        double L = (double)order * lambda / n2v / s.gr_const;
        return diffract<Sh>(s, mu, L, r) ? ACT_OK : ACT_LOST;
    }
    return ACT_OK;
}

}  // namespace f64
}  // namespace rtb
