// dual.cuh -- forward-mode dual numbers for the adjoint kernels.
//
// Dual<W> carries a value and W tangents.  The value is computed with the
// same IEEE operation as plain double arithmetic (translation units that use
// it are compiled with --fmad=false), so a trace in Dual<W> has exactly the
// values of the plain FP64 engine; the tangents follow the chain rule.
#pragma once

#include <cmath>

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
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
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
template <int W>
__device__ __forceinline__ Dual<W> operator/(const Dual<W>& a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a.v / b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator/(const Dual<W>& a, double b) {
    Dual<W> r;
    r.v = a.v / b;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = a.d[i] / b;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> operator/(double a, const Dual<W>& b) {
    Dual<W> r;
    r.v = a / b.v;
#pragma unroll
    for (int i = 0; i < W; ++i) r.d[i] = -r.v * b.d[i] / b.v;
    return r;
}
template <int W>
__device__ __forceinline__ Dual<W> sqrt(const Dual<W>& a) {
    Dual<W> r;
    r.v = ::sqrt(a.v);
    const double h = (r.v > 0.0) ? 0.5 / r.v : 0.0;
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
