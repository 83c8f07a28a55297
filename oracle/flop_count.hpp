// flop_count.hpp -- an operation-counting scalar for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (like rt_oracle.hpp).  Flop carries the double
// value the oracle computes -- so every comparison, loop and branch of the
// reference's algorithm goes exactly as in the FP64 oracle -- and counts the
// floating-point operations it performs: add, subtract, multiply, divide and
// square root 1 each (a fused multiply-add, which the reference's source does
// not write, would be 2), comparisons, negation and absolute value 0.
// Instantiating the oracle's per-ray functions (rt_oracle.hpp) on Flop gives
// the algorithmic operation count of the reference's per-ray arithmetic
// (cuda_engine/rt_cuda_engine_surface.cu kernel bodies, Beam::Normalize,
// ApplyConstrains, TabulatedFunction::operator[]), which is the numerator of
// the engine's compute roofline.
#pragma once

#include <cmath>
#include <cstdint>

namespace rto {

struct Flop {
    double v = 0.0;
    Flop() = default;
    Flop(double x) : v(x) {}  // NOLINT: constants and data enter the count as operands
    static thread_local uint64_t n;  // operations counted on this thread
};

inline thread_local uint64_t Flop::n = 0;

inline Flop operator+(Flop a, Flop b) { ++Flop::n; return Flop(a.v + b.v); }
inline Flop operator-(Flop a, Flop b) { ++Flop::n; return Flop(a.v - b.v); }
inline Flop operator*(Flop a, Flop b) { ++Flop::n; return Flop(a.v * b.v); }
inline Flop operator/(Flop a, Flop b) { ++Flop::n; return Flop(a.v / b.v); }
inline Flop operator-(Flop a) { return Flop(-a.v); }
inline Flop& operator+=(Flop& a, Flop b) { a = a + b; return a; }
inline Flop& operator-=(Flop& a, Flop b) { a = a - b; return a; }
inline Flop& operator*=(Flop& a, Flop b) { a = a * b; return a; }
inline Flop& operator/=(Flop& a, Flop b) { a = a / b; return a; }
inline bool operator<(Flop a, Flop b) { return a.v < b.v; }
inline bool operator>(Flop a, Flop b) { return a.v > b.v; }
inline bool operator<=(Flop a, Flop b) { return a.v <= b.v; }
inline bool operator>=(Flop a, Flop b) { return a.v >= b.v; }
inline bool operator==(Flop a, Flop b) { return a.v == b.v; }
inline bool operator!=(Flop a, Flop b) { return a.v != b.v; }
inline Flop sqrt(Flop a) { ++Flop::n; return Flop(std::sqrt(a.v)); }
inline Flop fabs(Flop a) { return Flop(std::fabs(a.v)); }

}  // namespace rto
