// adjoint_rev.cuh -- the adjoint's forward with checkpoints, its reverse
// sweep and its forward-mode sensitivities, as the bodies of the generic
// kernels (k_adj_forward, k_adj_reverse, k_adj_jvp, adjoint.cu) and of
// kernels compiled for one scheme's structure (jit.cpp,
// rtb_adj_forward_scheme, rtb_adj_reverse_scheme, rtb_adj_jvp_scheme).
//
// Forward: the fused FP64 engine's per-ray loop (the same bits), storing each
// ray's state (X Y Z cX cY cZ) at the input of every surface -- 48 bytes x
// surfaces per ray.
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

// Surface k (structure Sh) of the forward on one ray: its input state
// stored as checkpoint k, then the plain FP64 engine's surface.  -1 while
// the ray survives, the stage that lost it, or -2 (a wavelength outside a
// table).
template <class Sh>
__device__ __forceinline__ int fwd_surface(const AdjArgs& a, int k, size_t i, int b, double lam, unsigned* err,
                                           f64::Ray& r) {
    double* c = a.ckpt + (size_t)k * 6 * a.n + i;
    c[0] = r.X;
    c[a.n] = r.Y;
    c[2 * a.n] = r.Z;
    c[3 * a.n] = r.cX;
    c[4 * a.n] = r.cY;
    c[5 * a.n] = r.cZ;
    const DevScheme* sch = a.sch;
    const DevSurface& s = sch->s[k];
    f64::transform<Sh>(s, r);
    f64::normalize(r.cX, r.cY, r.cZ);
    if (!Sh::non_aux(s)) return -1;
    if (!f64::intersect<Sh>(s, sch->fixes, r)) return 3 * k;
    if (!f64::aperture_pass(Sh::type(s) == RTB_SHADE, Sh::shape(s), s.size, s.center, r.X, r.Y)) return 3 * k + 1;
    const int act = f64::action<Sh>(s, a.knots, adj_order(s, a.beams, b), lam, r);
    if (act == f64::ACT_RANGE) {
        atomicOr(err, DEV_ERR_OUT_OF_RANGE);
        return -2;
    }
    if (act == f64::ACT_LOST) return 3 * k + 2;
    f64::normalize(r.cX, r.cY, r.cZ);
    return -1;
}

// The forward through any scheme, its structure read at run time.
struct RtAdjForward {
    __device__ __forceinline__ static int run(const AdjArgs& a, size_t i, int b, double lam, unsigned* err,
                                              f64::Ray& r) {
        int stage = -1;
        for (int k = 0; k < a.sch->n_surfaces && stage == -1; ++k) stage = fwd_surface<RtShape>(a, k, i, b, lam, err, r);
        return stage;
    }
};

// in: the rays; counts: [n_beams][3 n_surfaces + 1] loss and arrival counters.
template <class Surfaces>
__device__ __forceinline__ void adj_forward(const AdjArgs& a, const DevRays& in, unsigned long long* counts,
                                            unsigned* err) {
    const int n_stages = 3 * a.sch->n_surfaces;
    for (size_t i = gtid(); i < a.n; i += gstride()) {
        a.lambda[i] = in.lambda[i];
        if (in.flag[i] != 1) {
            a.flag[i] = 0;
            continue;
        }
        f64::Ray r{in.X[i], in.Y[i], in.Z[i], in.cX[i], in.cY[i], in.cZ[i]};
        const double lam = in.lambda[i];
        const int b = beam_of(a.beams, a.n_beams, i);
        const int stage = Surfaces::run(a, i, b, lam, err, r);
        a.flag[i] = (stage == -1) ? 1 : 0;
        a.X[i] = r.X;
        a.Y[i] = r.Y;
        // one atomic per distinct counter in the warp (the rays of a beam
        // mostly share theirs)
        count_event(stage != -2, b * (n_stages + 1) + (stage >= 0 ? stage : n_stages), counts);
    }
}

// Surface k (structure Sh) of the forward-mode sensitivities on one ray:
// table[k] holds the surface's constants along the direction.
template <class Sh>
__device__ __forceinline__ void jvp_surface(const AdjArgs& a, int k, const ad::SurfD<1>* table, int b, double lam,
                                            ad::RayD<1>& r) {
    const DevSurface& s = a.sch->s[k];
    ad::surface_step<1, Sh>(s, table[k], a.sch->fixes, a.knots, adj_order(s, a.beams, b), lam, r);
}

// The sensitivities through any scheme, its structure read at run time.
struct RtAdjJvp {
    __device__ __forceinline__ static void run(const AdjArgs& a, const ad::SurfD<1>* table, int b, double lam,
                                               ad::RayD<1>& r) {
        for (int k = 0; k < a.sch->n_surfaces; ++k) jvp_surface<RtShape>(a, k, table, b, lam, r);
    }
};

// dX, dY: the rays' CCD-position sensitivities along the direction whose
// surface constants table[k] holds, through the whole scheme from the
// entrance rays (checkpoint 0); 0 for lost rays.
template <class Surfaces>
__device__ __forceinline__ void adj_jvp(const AdjArgs& a, const ad::SurfD<1>* table, double* dX, double* dY) {
    for (size_t i = gtid(); i < a.n; i += gstride()) {
        if (a.flag[i] != 1) {
            dX[i] = 0.0;
            dY[i] = 0.0;
            continue;
        }
        const double lam = a.lambda[i];
        const int b = beam_of(a.beams, a.n_beams, i);
        ad::Seeds<1> sd;
        sd.dense = nullptr;
        sd.state[0] = -1;
        sd.param[0] = -1;
        double st[6];
        for (int c = 0; c < 6; ++c) st[c] = a.ckpt[(size_t)c * a.n + i];
        ad::RayD<1> r;
        ad::load_state(st, sd, r);
        Surfaces::run(a, table, b, lam, r);
        dX[i] = r.X.d[0];
        dY[i] = r.Y.d[0];
    }
}

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
