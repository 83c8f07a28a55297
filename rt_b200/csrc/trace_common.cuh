// trace_common.cuh -- device helpers shared by the trace kernels.
#pragma once

#include "kernels.cuh"

namespace rtb {

__device__ __forceinline__ size_t gtid() { return (size_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ size_t gstride() { return (size_t)blockDim.x * gridDim.x; }

// Count one event per lane that has `pred`, one atomic per warp.
__device__ __forceinline__ void warp_count(bool pred, unsigned long long* counter) {
    unsigned mask = __ballot_sync(__activemask(), pred);
    if (pred && (threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1)) atomicAdd(counter, (unsigned long long)__popc(mask));
}

// __double2uint_rz: round toward zero, saturating, NaN -> 0 (rt_cuda_engine_ccd.cu:37-38).
__device__ __forceinline__ void ccd_coords(double X, double Y, double xsize, double ysize, double xpix, double ypix,
                                           unsigned& ix, unsigned& iy) {
    ix = __double2uint_rz((X + xsize / 2.0) / xpix);
    iy = __double2uint_rz((Y + ysize / 2.0) / ypix);
}

// Work distribution of the persistent fused kernels: a warp takes the next
// tile of 32*rpt consecutive rays from a global counter (zeroed before the
// launch) until the rays run out, so warps whose rays were lost early take
// more tiles and the grid drains evenly.  Ray j*32 + lane of a tile belongs
// to lane `lane`, which keeps every load and store of the tile coalesced.
__device__ __forceinline__ bool next_tile(const TileSched& ts, uint64_t n_tiles, uint64_t& tile) {
    unsigned long long t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(ts.next, 1ull);
    tile = __shfl_sync(0xffffffffu, t, 0);
    return tile < n_tiles;
}

__device__ __forceinline__ int beam_of(const DevBeam* beams, int n_beams, uint64_t i) {
    int lo = 0, hi = n_beams - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (beams[mid].first_ray <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// What the surfaces need of a ray's beam, read once per beam (BeamCursor):
// whether the beam sets the gratings' orders, the orders of the first two
// gratings (further ones are read from the table), and the beam's entry for
// the FP32-state engine's first-surface offset.
struct BeamCtx {
    const DevBeam* bm;
    long long ord0, ord1;
    bool per_beam;
    __device__ __forceinline__ long long order(const DevSurface& s) const {
        if (!per_beam) return s.order;
        const int g = s.grating_index;
        return g == 0 ? ord0 : (g == 1 ? ord1 : bm->orders[g]);
    }
};

__device__ __forceinline__ BeamCtx beam_ctx(const DevBeam* beams, int b) {
    const DevBeam& d = beams[b];
    return BeamCtx{&d, d.orders[0], d.orders[1], d.n_orders > 0};
}

// The beam of the rays being traced and what the surfaces need of it,
// cached per thread: rays come in increasing order (of index, or of slot in
// a plan's beam-major order), so the beam of the previous ray is usually
// this one's, and the beam table is read only when a ray falls outside the
// cached beam's range.
struct BeamCursor {
    int b = 0;
    uint64_t lo = 1, hi = 0;  // empty: the first ray searches
    BeamCtx ctx{nullptr, 0, 0, false};
    __device__ __forceinline__ int at(const DevBeam* beams, int n_beams, uint64_t i) {
        if (i < lo || i >= hi) {
            b = beam_of(beams, n_beams, i);
            lo = (b == 0) ? 0ull : beams[b].first_ray;
            hi = (b + 1 < n_beams) ? beams[b + 1].first_ray : ~0ull;
            ctx = beam_ctx(beams, b);
        }
        return b;
    }
};

// Count one event per lane (a loss at a stage, or reaching the end), one
// atomic per distinct counter in the warp.
__device__ __forceinline__ void count_event(bool ev, int key, unsigned long long* counts) {
    unsigned active = __activemask();
    unsigned em = __ballot_sync(active, ev);
    if (!ev) return;
    unsigned same = __match_any_sync(em, key);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(same) - 1)) atomicAdd(counts + key, (unsigned long long)__popc(same));
}

// Frame counts of one good ray at the detector: warp-aggregated increments
// of the pixel it lands on.  Non-finite coordinates count as outside.  The
// FP64 kernels divide by the pixel size as the reference does; the mixed
// kernel (kDivide false) multiplies by its reciprocal, which moves a ray to
// the next pixel only when its coordinate lies within an ulp of a pixel edge,
// and saves two FP64 division sequences per ray.
template <bool kDivide = true>
__device__ __forceinline__ void frame_add(bool good, double X, double Y, const FrameArgs& f) {
    unsigned active = __activemask();
    long long pix = -1;
    if (good) {
        if (isfinite(X) && isfinite(Y)) {
            unsigned ix, iy;
            if (kDivide) {
                ccd_coords(X, Y, f.xsize, f.ysize, f.xpix, f.ypix, ix, iy);
            } else {
                ix = __double2uint_rz((X + 0.5 * f.xsize) * f.inv_xpix);
                iy = __double2uint_rz((Y + 0.5 * f.ysize) * f.inv_ypix);
            }
            if (ix < f.xdim && iy < f.ydim) pix = (long long)iy * (long long)f.xdim + ix;
        }
    }
    bool in = pix >= 0;
    unsigned im = __ballot_sync(active, in);
    if (in) {
        unsigned same = __match_any_sync(im, pix);
        if ((threadIdx.x & 31) == (unsigned)(__ffs(same) - 1)) atomicAdd(f.counts + pix, (unsigned)__popc(same));
    }
    bool out = good && !in;
    unsigned om = __ballot_sync(active, out);
    if (out && f.n_outside && (threadIdx.x & 31) == (unsigned)(__ffs(om) - 1))
        atomicAdd(f.n_outside, (unsigned long long)__popc(om));
}

// Copy the scheme and the knot tables into shared memory (fused kernels).
__device__ __forceinline__ const DevScheme* stage_scheme(const DevScheme* sch, const double* knots,
                                                         const double*& s_knots) {
    extern __shared__ __align__(16) unsigned char smem[];
    DevScheme* s_sch = reinterpret_cast<DevScheme*>(smem);
    double* kn = reinterpret_cast<double*>(smem + ((sizeof(DevScheme) + 15) / 16) * 16);
    const int4* src = reinterpret_cast<const int4*>(sch);
    int4* dst = reinterpret_cast<int4*>(smem);
    for (int j = threadIdx.x; j < (int)(sizeof(DevScheme) / 16); j += blockDim.x) dst[j] = src[j];
    int nk = sch->n_knots;
    for (int j = threadIdx.x; j < nk; j += blockDim.x) kn[j] = knots[j];
    __syncthreads();
    s_knots = kn;
    return s_sch;
}

}  // namespace rtb
