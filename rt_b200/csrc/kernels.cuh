// kernels.cuh -- kernel declarations and their argument structs.
#pragma once

#include "common.cuh"

namespace rtb {

// One beam for the generator (rtb_generate_beams).
struct GenBeam {
    uint64_t first_ray, n_rays, n_lambda;
    uint64_t seed;
    double disk[3];     // N, R_in, R_out
    double center[3];
    double range[2];
    double d_lambda;    // (range[1]-range[0])/(n_lambda-1) (rt_cuda_engine_beam.cu:726)
    double c0[3];       // direction cosines of the field angle, normalised
};

// CCD frame accumulation arguments.
struct FrameArgs {
    double xsize, ysize, xpix, ypix;
    uint64_t xdim, ydim;
    unsigned* counts;               // device; NULL disables the frame
    unsigned long long* n_outside;  // device; may be NULL
    double inv_xpix, inv_ypix;      // 1/xpix, 1/ypix (the mixed kernel's pixel coordinates)
};

#ifndef __CUDACC_RTC__
// Size of the dynamic shared memory the fused kernels use.
inline size_t fused_smem_bytes(int n_knots) {
    return ((sizeof(DevScheme) + 15) / 16) * 16 + sizeof(double) * (size_t)n_knots;
}
#endif

// Scheduling of the persistent fused kernels: `next` is a counter of tiles
// (zeroed before each launch) handed out to warps, 32*rpt rays each (the
// mixed kernels), or to blocks, blockDim*rpt rays each (k_fused_fp64).  Slot
// s of the tiles traces ray order[s] (a permutation of the rays), or ray s
// when order is NULL; its input is read at s when in_by_slot (the input
// arrays hold the rays in tracing order), else at the ray's index.  Outputs
// go to the ray's index unless out_by_slot.
// `rows` (mixed kernels, may be NULL): the rays in tracing order as row
// blocks (Row64 for RTB_MIXED, Row32 for RTB_MIXED32, rowpipe.cuh), read in
// place of `in`.  out_by_slot: outputs go to the tracing slot instead.
struct TileSched {
    unsigned long long* next;
    int rpt;
    const uint32_t* order;
    int in_by_slot;
    const void* rows;
    int out_by_slot;
};
constexpr int kDefaultRpt = 2;

// One surface of a throughput curve (k_qe_curves): its QE table in the knot
// array, and for a grating the order and rule parameters, angles in radians.
struct QeSurface {
    int32_t off, cnt;
    int32_t grating;
    int32_t pad;
    long long order;
    double gr_const, alpha, gamma, blaze, rule_size;
};

// ---- drop-in kernels (kernels_fp64.cu) ----
__global__ void k_transform(size_t n, DevSurface s, double* X, double* Y, double* Z, double* cX, double* cY,
                            double* cZ);
__global__ void k_intersect(size_t n, DevSurface s, uint32_t fixes, double* X, double* Y, double* Z,
                            const double* cX, const double* cY, const double* cZ, char* flag,
                            unsigned long long* n_bad);
__global__ void k_reflect(size_t n, DevSurface s, const double* X, const double* Y, const double* Z, double* cX,
                          double* cY, double* cZ);
__global__ void k_action(size_t n, DevSurface s, const double* knots, long long order, const double* lambda,
                         const double* X, const double* Y, const double* Z, double* cX, double* cY, double* cZ,
                         char* flag, unsigned long long* n_bad, unsigned* err);
__global__ void k_normalize(size_t n, double* cX, double* cY, double* cZ);
__global__ void k_aperture(size_t n, int shade, int shape, double sz0, double sz1, double c0, double c1,
                           const double* X, const double* Y, char* flag, unsigned long long* n_bad);
__global__ void k_ccd_coords(size_t n, const double* X, const double* Y, double xsize, double ysize, double xpix,
                             double ypix, unsigned* ix, unsigned* iy);
__global__ void k_ccd_image(size_t n, const unsigned* ix, const unsigned* iy, const double* lambda,
                            const double* knots, int qe_off, int qe_n, int sp_off, int sp_n, size_t xdim, size_t ydim,
                            double pix_area, double* image, unsigned long long* n_outside, unsigned* err);
__global__ void k_surface_qe(size_t n, const double* lambda, double* spec, const double* knots, int off, int cnt,
                             unsigned* err);
__global__ void k_qe_curves(size_t n_lambda, size_t n_rows, const double* rows, size_t row_len, const QeSurface* s,
                            int n_s, const double* knots, int orders_from_rows, double* lambda, double* qe,
                            unsigned* err);
__global__ void k_beam_random(size_t n, double p1, double p2, double cx, double cy, double cz, uint64_t seed,
                              uint64_t first, double* X, double* Y, double* Z);
__global__ void k_uniform_range(size_t n, double l0, double d_l, double* lambda);
__global__ void k_random_range(size_t n, double l0, double l1, uint64_t seed, double* lambda);
__global__ void k_generate(const GenBeam* beams, int n_beams, uint64_t total, DevRays rays);
// order.cu: sort keys of the coherent tracing order of generated rays
__global__ void k_order_keys(const GenBeam* beams, int n_beams, uint64_t total, DevRays rays,
                             unsigned long long* keys, uint32_t* idx, int chunk_shift);
// dst[s] = src[order[s]] for X..lambda and flag
__global__ void k_gather_rays(const uint32_t* order, uint64_t n, DevRays src, DevRays dst);
// the same into row blocks of 32 rays (rowpipe.cuh): FP64 (Row64), or FP32
// positions relative to the beam's origin and FP32 cosines (Row32); slots
// past n up to a whole row get flag 0
__global__ void k_gather_rows64(const uint32_t* order, uint64_t n, DevRays src, void* rows);
__global__ void k_gather_rows32(const uint32_t* order, uint64_t n, DevRays src, const DevBeam* beams, int n_beams,
                                void* rows);
__global__ void k_ccd_frame(DevRays rays, FrameArgs f);

// ---- trace kernels ----
// counts: [n_beams][3*n_surfaces + 1] -- rays lost per stage, then rays that
// reached the end.
// Rays are read from `in` and written to `out` (which may be `in`); a lost
// ray's flag and lost_stage are written to `out`.
__global__ void k_surface_step(const DevScheme* sch, int k, const double* knots, const DevBeam* beams, int n_beams,
                               DevRays in, DevRays out, unsigned long long* counts, unsigned* err);
__global__ void k_fused_fp64(const DevScheme* sch, const double* knots, const DevBeam* beams, int n_beams,
                             DevRays in, DevRays out, unsigned long long* counts, unsigned* err, int state_out,
                             FrameArgs frame, TileSched ts);
// kernels_mixed.cu: FP64 state (RTB_MIXED) and FP32 state (RTB_MIXED32)
__global__ void k_fused_mixed32(const DevScheme* sch, const double* knots, const DevBeam* beams, int n_beams,
                                DevRays in, DevRays out, unsigned long long* counts, unsigned* err, int state_out,
                                FrameArgs frame, TileSched ts);
__global__ void k_fused_mixed(const DevScheme* sch, const double* knots, const DevBeam* beams, int n_beams,
                              DevRays in, DevRays out, unsigned long long* counts, unsigned* err, int state_out,
                              FrameArgs frame, TileSched ts);

#ifndef __CUDACC_RTC__
// ---- ordering (order.cu) ----
int reference_order(const DevBeam* h_beams, int n_beams, int n_stages, const DevRays& rays, uint32_t* order,
                    cudaStream_t stream);
int rearrange_device(size_t n_good, double* arrays[7], char* flag, size_t* n_good_out, cudaStream_t stream);

#endif

}  // namespace rtb
