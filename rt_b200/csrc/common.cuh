// common.cuh -- device-side definitions shared by the engine's kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rtb.h"

namespace rtb {

// Constants of the reference (common-lib/num_defs.h:20,31;
// cuda_engine/rt_cuda_engine_beam.cu:41; rt_cuda_engine_ccd.cu:19;
// rt_cuda_engine_surface.cu:667-668).
constexpr double K_RT_PI = 3.14159265359;
constexpr double K_DEG2RAD = K_RT_PI / 180.0;   // value of `deg2rad` after *= or /=
constexpr double K_PI2 = 6.28318531;
constexpr double K_HC = 1.98644560233e-12;
constexpr double K_ITER_EPS = 1.0e-7;
constexpr unsigned K_ITER_MAX = 100000;

// Intersection algorithm of a surface, as engine_intersection_cycle picks it
// (rt_cuda_engine_surface.cu:593-636).
enum IsectKind : int32_t { IS_NONE = 0, IS_PLANE, IS_PARABOLOID, IS_CONIC, IS_ITER_POLY, IS_ITER_CONIC, IS_TORIC };

// Error bits a kernel raises for the host (the reference throws instead).
// DEV_ERR_TIMEOUT: a bounded wait of a kernel ran out (the staged copy of a
// ray row never completed); the call fails with RTB_FAILED.
enum DevError : uint32_t { DEV_ERR_OUT_OF_RANGE = 1u, DEV_ERR_BAD_VALUE = 2u, DEV_ERR_TIMEOUT = 4u };

// One surface as the kernels consume it: everything the reference's host
// code derives before a kernel launch (copy_surf_params, the transform's
// sin/cos, grating/lens constants) is precomputed on the host.
struct DevSurface {
    int32_t cls, type, shape, gr_type;
    int32_t kind;           // IsectKind
    int32_t grating_index;  // -1 unless a grating
    int32_t non_aux;
    int32_t renorm_after;   // Normalize calls that follow this surface's action
    int32_t surfaces_upto;  // non-Aux surfaces up to and including this one
    int32_t n_poly;
    int32_t translate;
    int32_t rot_mask;       // bit i: rotation i (about y, x, z) applies
    int64_t order;
    double gr_const;
    double c, k1, cR;
    double poly[RTB_MAX_POLY];
    double dist[3];
    double sinA[3], cosA[3];
    double size[2], center[2];
    int32_t n1_off, n1_n, n2_off, n2_n;  // tables: offset/count into the knot buffer (count 1 = single value)
    double n1_invh, n2_invh;              // 1/knot spacing of a table on a uniform grid, else 0 (mixed engine)
    // Even asphere with a circular pass aperture (mixed engine): every point of
    // the surface inside the aperture has sag_lo <= Z <= sag_hi.
    double sag_lo, sag_hi;
    int32_t sag_cull;                     // 1: sag_lo / sag_hi are set
    int32_t sag_pad;
    // 1/c and 1/gr_const (0 where c or gr_const is 0): the mixed engine
    // multiplies by them where the plain engine divides
    double inv_c, inv_gr;
    // FP32 copies for the mixed engine's normals and Newton derivatives:
    // c, k1, cR, 1/c, the polynomial coefficients a_i and i * a_i
    float f_c, f_k1, f_cR, f_inv_c;
    float f_poly[RTB_MAX_POLY], f_ipoly[RTB_MAX_POLY];
    float f_sag_lo, f_sag_hi, f_size0, f_pad;  // sag range and aperture radius
    // FP32-state engine (RTB_MIXED32): the transform from the frame of the
    // previous non-Aux surface (the entrance frame for the first), with the
    // Aux surfaces in between folded in, as P' = M P + off32 and D' = M D:
    // M in FP32 (rows), off32 in FP64.  rot32: M is not the identity;
    // first32: the first non-Aux surface, whose offset comes from the ray's
    // beam (DevBeam::off0).  Set on non-Aux surfaces only.  Each entry of M is
    // held twice, (m, m): the operand pair of the paired FP32 multiply-adds
    // that rotate a position and a direction cosine together.
    float2 m32[9];
    int32_t rot32, first32, pad32;
    double off32[3];
};

// A prepared scheme in device memory; the fused kernels copy it to shared
// memory, the per-surface kernel reads its one surface from global memory.
struct DevScheme {
    int32_t n_surfaces;
    int32_t n_knots;        // doubles per array in the knot buffer
    uint32_t fixes;
    int32_t renorm_lost;
    int32_t pad[4];
    DevSurface s[RTB_MAX_SURFACES];
    // FP32-state engine: the first non-Aux surface's transform in FP64 (from
    // the entrance frame), from which each beam's offset is made, and the
    // transform of the Aux surfaces after the last non-Aux one (tail_on).
    double m0[9], off0[3];
    double tail_m[9], tail_off[3];
    int32_t tail_on, pad_tail[3];
};
static_assert(sizeof(DevScheme) % 16 == 0, "DevScheme is copied to shared memory in 16-byte words");

// Beam table on the device (first ray and orders of each beam).
struct DevBeam {
    uint64_t first_ray;
    uint64_t n_rays;
    int64_t orders[RTB_MAX_GRATINGS];
    int32_t n_orders;
    int32_t pad;
    // FP32-state engine: the beam's origin (rtb_beam::center), to which its
    // rays' FP32 positions are relative, and the offset of the first non-Aux
    // surface's transform for those positions (DevScheme m0 origin + off0)
    double origin[3], off0[3];
};

struct DevRays {
    double *X, *Y, *Z, *cX, *cY, *cZ, *lambda;
    char* flag;
    uint8_t* lost_stage;
    uint64_t n;
};

}  // namespace rtb

#ifndef __CUDACC_RTC__  // host code (not in run-time compiled kernels)
#define RTB_CUDA_TRY(expr)                              \
    do {                                                \
        cudaError_t _e = (expr);                        \
        if (_e != cudaSuccess) return rtb::cuda_status(_e); \
    } while (0)

namespace rtb {
inline int cuda_status(cudaError_t e) {
    return (e == cudaErrorMemoryAllocation) ? RTB_BAD_ALLOC : RTB_FAILED;
}
}  // namespace rtb
#endif
