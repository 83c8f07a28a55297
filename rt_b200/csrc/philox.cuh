// philox.cuh -- the seeded synthetic beam generator (device side).
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11) gives two uniforms per ray; the uniform disk
// position follows random_circle_kernel (rt_cuda_engine_beam.cu:126-152).
// sin/cos use a Cody-Waite reduction (Cody & Waite, "Software Manual for the
// Elementary Functions", 1980) and Taylor polynomials evaluated with plain
// IEEE operations, so that the beam is bit-identical to the CPU oracle's
// generator (the translation unit is compiled with --fmad=false).
#pragma once

#include <cstdint>

namespace rtb {

struct U4 {
    uint32_t v[4];
};

__device__ __forceinline__ U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        uint32_t lo0 = M0 * ctr.v[0], hi0 = __umulhi(M0, ctr.v[0]);
        uint32_t lo1 = M1 * ctr.v[2], hi1 = __umulhi(M1, ctr.v[2]);
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

// Uniform double in (0,1]: ((b >> 11) + 1) * 2^-53.
__device__ __forceinline__ double u01_from_bits(uint32_t hi, uint32_t lo) {
    uint64_t b = ((uint64_t)hi << 32) | lo;
    return (double)((b >> 11) + 1) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ void ray_uniforms(uint64_t seed, uint64_t stream, uint64_t ray, double& u1, double& u2) {
    U4 c;
    c.v[0] = (uint32_t)ray;
    c.v[1] = (uint32_t)(ray >> 32);
    c.v[2] = (uint32_t)stream;
    c.v[3] = (uint32_t)(stream >> 32);
    U4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    u1 = u01_from_bits(r.v[0], r.v[1]);
    u2 = u01_from_bits(r.v[2], r.v[3]);
}

// sin and cos for |x| < 1e5 (the generator calls it on [0, 2*pi)).
__device__ __forceinline__ void beam_sincos(double x, double& s, double& c) {
    const double INV_PIO2 = 0.6366197723675814;
    const double P1 = 1.5707963267341256e+00;
    const double P2 = 6.077100506303966e-11;
    const double P3 = 2.0222662487959506e-21;
    double k = rint(x * INV_PIO2);
    double r = ((x - k * P1) - k * P2) - k * P3;
    double r2 = r * r;
    double ps = 1.0 / 121645100408832000.0;
    ps = ps * (-r2) + 1.0 / 355687428096000.0;
    ps = ps * (-r2) + 1.0 / 1307674368000.0;
    ps = ps * (-r2) + 1.0 / 6227020800.0;
    ps = ps * (-r2) + 1.0 / 39916800.0;
    ps = ps * (-r2) + 1.0 / 362880.0;
    ps = ps * (-r2) + 1.0 / 5040.0;
    ps = ps * (-r2) + 1.0 / 120.0;
    ps = ps * (-r2) + 1.0 / 6.0;
    ps = ps * (-r2) + 1.0;
    double sr = r * ps;
    double pc = 1.0 / 2432902008176640000.0;
    pc = pc * (-r2) + 1.0 / 6402373705728000.0;
    pc = pc * (-r2) + 1.0 / 20922789888000.0;
    pc = pc * (-r2) + 1.0 / 87178291200.0;
    pc = pc * (-r2) + 1.0 / 479001600.0;
    pc = pc * (-r2) + 1.0 / 3628800.0;
    pc = pc * (-r2) + 1.0 / 40320.0;
    pc = pc * (-r2) + 1.0 / 720.0;
    pc = pc * (-r2) + 1.0 / 24.0;
    pc = pc * (-r2) + 1.0 / 2.0;
    double cr = 1.0 - r2 * pc;
    switch ((long long)k & 3) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}

// params = [N, R_in, R_out], center = [x, y, z]
__device__ __forceinline__ void disk_position(const double* params, const double* center, double u1, double u2,
                                              double& X, double& Y, double& Z) {
    const double PI2 = 6.28318531;
    double phi = PI2 * u2;
    Z = center[2];
    double R = (params[2] - params[1]) * sqrt(u1) + params[1];
    double sp, cp;
    beam_sincos(phi, sp, cp);
    X = R * cp + center[0];
    Y = R * sp + center[1];
}

}  // namespace rtb
