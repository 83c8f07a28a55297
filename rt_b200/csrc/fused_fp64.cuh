// fused_fp64.cuh -- device code of the fused FP64 trace kernel.
//
// Bit-identical to the per-surface engine (ray_fp64.cuh; compiled with
// --fmad=false): k_fused_fp64 runs it for any scheme, reading each surface's
// structure at run time; a plan of a fixed scheme launches a copy compiled
// for that scheme's structure (jit.cpp), which executes the same IEEE
// operations in the same order.
#pragma once

#include "trace_common.cuh"
#include "ray_fp64.cuh"

namespace rtb {

// One surface of the fused FP64 trace on one live ray: transform, Normalize,
// intersection, aperture, action, Normalize; `stage` becomes the stage that
// lost the ray, or -2 for a wavelength outside a table.
template <class Sh = RtShape>
__device__ __forceinline__ void f64_surface(const DevSurface& s, int k, uint32_t fixes, const double* knots,
                                            const DevBeam* beams, int b, double lam, unsigned* err, f64::Ray& r,
                                            int& stage) {
    f64::transform<Sh>(s, r);
    f64::normalize(r.cX, r.cY, r.cZ);
    if (!Sh::non_aux(s)) return;
    if (!f64::intersect<Sh>(s, fixes, r)) {
        stage = 3 * k;
    } else if (!f64::aperture_pass(Sh::type(s) == RTB_SHADE, Sh::shape(s), s.size, s.center, r.X, r.Y)) {
        stage = 3 * k + 1;
    } else {
        long long order = s.order;
        if (Sh::type(s) == RTB_GRATING && beams[b].n_orders > 0) order = beams[b].orders[s.grating_index];
        int a = f64::action<Sh>(s, knots, order, lam, r);
        if (a == f64::ACT_RANGE) {
            atomicOr(err, DEV_ERR_OUT_OF_RANGE);
            stage = -2;
        } else if (a == f64::ACT_LOST) {
            stage = 3 * k + 2;
        } else {
            f64::normalize(r.cX, r.cY, r.cZ);
        }
    }
}

// The surfaces in order, the whole block stepping through them together (a
// barrier after each; every thread calls run, also without a live ray).
struct RtSurfacesF64 {
    __device__ __forceinline__ static void run(const DevScheme* sch, const double* knots, const DevBeam* beams,
                                               int b, double lam, unsigned* err, f64::Ray& r, int& stage) {
        for (int k = 0; k < sch->n_surfaces; ++k) {
            if (stage == -1) f64_surface(sch->s[k], k, sch->fixes, knots, beams, b, lam, err, r, stage);
            __syncthreads();
        }
    }
};

// Fused FP64 trace: the whole surface sequence per ray in registers, the
// scheme and knot tables in shared memory, a persistent grid whose blocks
// take tiles of blockDim x rpt rays from the counter.  The block steps
// through the surfaces together (a barrier after each): the bit-exact code of
// all surface kinds is larger than the instruction cache, and warps spread
// over different surfaces missed it on most issues (ncu: 12 cycles of
// no_instruction stall per issued instruction, C1 29.8 ms); in step, one
// surface's code serves the whole block (24.5 ms).  Bit-identical to
// k_surface_step.  With a frame, good rays add their pixel with
// warp-aggregated atomics.
template <class Surfaces>
__device__ __forceinline__ void fused_fp64(const DevScheme* __restrict__ g_sch, const double* knots,
                                           const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                           unsigned long long* counts, unsigned* err, int state_out,
                                           FrameArgs frame, TileSched ts) {
    const double* s_knots;
    const DevScheme* sch = stage_scheme(g_sch, knots, s_knots);
    const int ns = sch->n_surfaces;
    const int n_stages = 3 * ns;
    const uint64_t block_rays = (uint64_t)blockDim.x * (uint64_t)ts.rpt;
    const uint64_t n_tiles = (in.n + block_rays - 1) / block_rays;
    __shared__ unsigned long long s_tile;
    int b = 0;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ts.next, 1ull);
        __syncthreads();
        const uint64_t tile = s_tile;
        __syncthreads();
        if (tile >= n_tiles) break;
        for (int j = 0; j < ts.rpt; ++j) {
            const size_t slot = tile * block_rays + (size_t)j * blockDim.x + threadIdx.x;
            const size_t i = (ts.order && slot < in.n) ? (size_t)ts.order[slot] : slot;
            const size_t ri = ts.in_by_slot ? slot : i;
            const size_t oi = ts.out_by_slot ? slot : i;  // where its results go
            bool ev = false, good = false;
            int key = 0;
            double outX = 0, outY = 0;
            const bool have = slot < in.n && in.flag[ri] == 1;
            f64::Ray r{0, 0, 0, 0, 0, 0};
            double lam = 0;
            if (have) {
                r = f64::Ray{in.X[ri], in.Y[ri], in.Z[ri], in.cX[ri], in.cY[ri], in.cZ[ri]};
                lam = in.lambda[ri];
                if (!(b + 1 >= n_beams || i < beams[b + 1].first_ray) || i < beams[b].first_ray)
                    b = beam_of(beams, n_beams, i);
            } else if (slot < in.n && in.flag != out.flag) {
                out.flag[oi] = in.flag[ri];
            }
            int stage = have ? -1 : -3;
            Surfaces::run(sch, s_knots, beams, b, lam, err, r, stage);
            if (have) {
                if (stage >= 0) {
                    ev = true;
                    if (sch->renorm_lost) f64::renormalize(r, sch->s[stage / 3].renorm_after);
                    out.flag[oi] = 0;
                    out.lost_stage[oi] = (uint8_t)stage;
                    key = b * (n_stages + 1) + stage;
                } else if (stage == -1) {
                    ev = good = true;
                    key = b * (n_stages + 1) + n_stages;
                    if (in.flag != out.flag) {
                        out.flag[oi] = 1;
                        out.lost_stage[oi] = RTB_NOT_LOST;
                    }
                }
                if (stage != -2) {
                    out.X[oi] = r.X;
                    out.Y[oi] = r.Y;
                    if (state_out) {
                        out.Z[oi] = r.Z;
                        out.cX[oi] = r.cX;
                        out.cY[oi] = r.cY;
                        out.cZ[oi] = r.cZ;
                    }
                }
                outX = r.X;
                outY = r.Y;
            }
            count_event(ev, key, counts);
            if (frame.counts) frame_add(good, outX, outY, frame);
        }
    }
}

}  // namespace rtb
