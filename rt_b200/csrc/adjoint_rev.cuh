// adjoint_rev.cuh -- the adjoint's reverse sweep, as the body of the generic
// kernel (k_adj_reverse, adjoint.cu) and of kernels compiled for one
// scheme's structure (jit.cpp, rtb_adj_reverse_scheme).
//
// Per ray, surfaces last to first: surface k is recomputed from checkpoint k
// and the adjoint of its output state is carried back through its stages in
// reverse order (ray_rev.cuh), giving the adjoint of its input state and of
// the constants its parameters move, in one sweep.  Rays are taken 32 at a
// time per warp, every lane of a warp the same number of steps, so the warp
// sums each parameter's contributions over its lanes with a shuffle tree
// into its row in shared memory; the block adds its warps' rows in order and
// writes one partial per parameter, which the caller sums in block order: the
// gradient is reproducible.
#pragma once

#include "ray_rev.cuh"
#include "trace_common.cuh"

namespace rtb {

constexpr int kAdjThreads = 128;
constexpr int kAdjWarps = kAdjThreads / 32;

struct AdjArgs {
    const DevScheme* sch;
    const double* knots;
    const DevBeam* beams;
    int n_beams;
    const ad::ParamRef* map;
    int n_params;
    const int* surf_params;  // [n_surfaces][RTB_ADJ_MAX_PARAMS]: parameter indices per surface
    const int* surf_nparams; // [n_surfaces]
    double* ckpt;            // [(k * 6 + c) * n + i]
    double* lambda;          // copy of the wavelengths
    char* flag;              // 1 = reached the end
    double* X;
    double* Y;
    uint64_t n;
};

// The diffraction order of grating s for a ray of beam b.
__device__ __forceinline__ long long adj_order(const DevSurface& s, const DevBeam* beams, int b) {
    long long order = s.order;
    if (s.type == RTB_GRATING && beams[b].n_orders > 0) order = beams[b].orders[s.grating_index];
    return order;
}

// A surface's structure as a kernel compiled for the adjoint's scheme reads
// it: fixed, except the translation and the rotations, which are read at run
// time -- a parameter may move a distance or an angle away from zero, and
// the recomputation must apply exactly the transforms the forward applied.
template <int KIND, int TYPE, int CLS, int SHAPE, int GRT, int NPOLY, int NONAUX, int POLYONLY>
struct AdjShape {
    __device__ __forceinline__ static constexpr int kind(const DevSurface&) { return KIND; }
    __device__ __forceinline__ static constexpr int type(const DevSurface&) { return TYPE; }
    __device__ __forceinline__ static constexpr int cls(const DevSurface&) { return CLS; }
    __device__ __forceinline__ static constexpr int shape(const DevSurface&) { return SHAPE; }
    __device__ __forceinline__ static constexpr int gr_type(const DevSurface&) { return GRT; }
    __device__ __forceinline__ static bool translate(const DevSurface& s) { return s.translate != 0; }
    __device__ __forceinline__ static int rot_mask(const DevSurface& s) { return s.rot_mask; }
    __device__ __forceinline__ static constexpr int n_poly(const DevSurface&) { return NPOLY; }
    __device__ __forceinline__ static constexpr bool non_aux(const DevSurface&) { return NONAUX != 0; }
    __device__ __forceinline__ static bool sag_cull(const DevSurface& s) { return s.sag_cull != 0; }
    __device__ __forceinline__ static constexpr bool poly_only(const DevSurface&) { return POLYONLY != 0; }
    __device__ __forceinline__ static bool rot32(const DevSurface& s) { return s.rot32 != 0; }
    __device__ __forceinline__ static bool first32(const DevSurface& s) { return s.first32 != 0; }
};

// One lane's ray in the reverse sweep.
struct RevRay {
    size_t i;
    bool act;       // traced to the end, with a seed
    int b;          // its beam
    double lam;
    rv::RayA adj;   // the adjoint of its state at the output of the next surface to sweep
};

// Surface k (structure Sh) of the reverse sweep for the warp's rays: the
// adjoint carried back through it, the contributions to its parameters
// summed over the warp into the warp's row of shared-memory sums.
template <class Sh>
__device__ __forceinline__ void rev_surface(const AdjArgs& a, int k, RevRay& ray, int lane, double* acc_row) {
    const DevScheme* sch = a.sch;
    const int np = a.surf_nparams[k];
    if (k == 0 && np == 0) return;  // the entrance rays' adjoint is not needed
    const DevSurface& s = sch->s[k];
    rv::SurfA pa;
    rv::clear(pa);
    if (ray.act) {
        const double* c = a.ckpt + (size_t)k * 6 * a.n + ray.i;
        const f64::Ray r0{c[0], c[a.n], c[2 * a.n], c[3 * a.n], c[4 * a.n], c[5 * a.n]};
        if (!rv::surface_rev<Sh>(s, sch->fixes, a.knots, adj_order(s, a.beams, ray.b), ray.lam, r0, ray.adj, pa)) {
            ray.act = false;  // not reached: the recomputation is the forward's
            rv::clear(pa);
        }
    }
    for (int q = 0; q < np; ++q) {
        const int j = a.surf_params[k * RTB_ADJ_MAX_PARAMS + q];
        double v = ray.act ? rv::param_adjoint(s, a.map[j], pa) : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) acc_row[j] += v;
    }
}

// The surfaces of any scheme, last to first, their structure read at run time.
struct RtAdjSurfaces {
    __device__ __forceinline__ static void sweep(const AdjArgs& a, RevRay& ray, int lane, double* acc_row) {
        for (int k = a.sch->n_surfaces - 1; k >= 0; --k) rev_surface<RtShape>(a, k, ray, lane, acc_row);
    }
};

// gX, gY: the adjoints of the rays' CCD positions; partial: [gridDim.x][n_params].
template <class Surfaces>
__device__ __forceinline__ void adj_reverse(const AdjArgs& a, const double* gX, const double* gY, double* partial) {
    __shared__ double acc[kAdjWarps][RTB_ADJ_MAX_PARAMS];
    const int P = a.n_params;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int p = lane; p < P; p += 32) acc[warp][p] = 0.0;
    __syncwarp();
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x + (size_t)warp * 32; i0 < a.n; i0 += gstride()) {
        RevRay ray;
        ray.i = i0 + lane;
        ray.act = ray.i < a.n && a.flag[ray.i] == 1;
        ray.adj = rv::RayA{ray.act ? gX[ray.i] : 0.0, ray.act ? gY[ray.i] : 0.0, 0.0, 0.0, 0.0, 0.0};
        ray.act = ray.act && !(ray.adj.X == 0.0 && ray.adj.Y == 0.0);
        if (!__any_sync(0xffffffffu, ray.act)) continue;
        ray.lam = ray.act ? a.lambda[ray.i] : 0.0;
        ray.b = ray.act ? beam_of(a.beams, a.n_beams, ray.i) : 0;
        Surfaces::sweep(a, ray, lane, acc[warp]);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        double sum = 0.0;
        for (int w = 0; w < kAdjWarps; ++w) sum += acc[w][p];
        partial[(size_t)blockIdx.x * P + p] = sum;
    }
}

}  // namespace rtb
