// dual.cuh -- forward-mode dual numbers for the adjoint kernels.
//
// Dual<W> carries a value and W tangents.  The value is computed with the
// same IEEE operation as plain double arithmetic (translation units that use
// it are compiled with --fmad=false), so a trace in Dual<W> has exactly the
// values of the plain FP64 engine; the tangents follow the chain rule with
// explicit fused multiply-adds (a product rule is one FMA and one multiply),
// their divisions as products with one refined reciprocal (tangent_rcp).
#pragma once

#ifndef __CUDACC_RTC__  // run-time compiled kernels take the device math built in
#include <cmath>
#endif

namespace rtb {
namespace ad {

template <int W>
struct Dual {
    double v;
    double d[W];
};

template <int W>
__device__ __forceinline__ Dual<W> cst(double v) {
    Dual<W> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = 0.0;
    return r;
}

template <int W>
__device__ __forceinline__ Dual<W> operator+(const Dual<W>& a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator+(const Dual<W>& a, double b) {
    Dual<W> r = a;
    r.v = a.v + b;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator+(double a, const Dual<W>& b) {
    Dual<W> r = b;
    r.v = a + b.v;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator-(const Dual<W>& a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator-(const Dual<W>& a, double b) {
    Dual<W> r = a;
    r.v = a.v - b;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator-(double a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a - b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = -b.d[i];
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator-(const Dual<W>& a) {
    Dual<W> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator*(const Dual<W>& a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = fma(a.d[i], b.v, a.v * b.d[i]);
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator*(const Dual<W>& a, double b) {
    Dual<W> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator*(double a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a * b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a * b.d[i];
    return r;
}
// 1/x for the tangents: the reciprocal seed refined by two Newton steps (to
// about an ulp).  The values keep IEEE division; a tangent's last bits do not
// steer anything, and one reciprocal per operation replaces W divisions.
__device__ __forceinline__ double tangent_rcp(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

template <int W>
__device__ __forceinline__ Dual<W> operator/(const Dual<W>& a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a.v / b.v;
    const double ib = tangent_rcp(b.v);
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = fma(-r.v, b.d[i], a.d[i]) * ib;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator/(const Dual<W>& a, double b) {
    Dual<W> r;
    r.v = a.v / b;
    const double ib = tangent_rcp(b);
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] * ib;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator/(double a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a / b.v;
    const double ib = tangent_rcp(b.v);
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = -r.v * b.d[i] * ib;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> sqrt(const Dual<W>& a) {
    Dual<W> r;
    r.v = ::sqrt(a.v);
    const double h = (r.v > 0.0) ? 0.5 * tangent_rcp(r.v) : 0.0;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] * h;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> fabs(const Dual<W>& a) {
    return (a.v < 0.0) ? -a : a;
}

template <int W> __device__ __forceinline__ Dual<W>& operator+=(Dual<W>& a, const Dual<W>& b) { return a = a + b; }
template <int W> __device__ __forceinline__ Dual<W>& operator-=(Dual<W>& a, const Dual<W>& b) { return a = a - b; }
template <int W> __device__ __forceinline__ Dual<W>& operator*=(Dual<W>& a, const Dual<W>& b) { return a = a * b; }
template <int W> __device__ __forceinline__ Dual<W>& operator/=(Dual<W>& a, const Dual<W>& b) { return a = a / b; }
template <int W> __device__ __forceinline__ Dual<W>& operator*=(Dual<W>& a, double b) { return a = a * b; }

// Comparisons and branches look at the value only.
template <int W> __device__ __forceinline__ double val(const Dual<W>& a) { return a.v; }
__device__ __forceinline__ double val(double a) { return a; }

}  // namespace ad
}  // namespace rtb
