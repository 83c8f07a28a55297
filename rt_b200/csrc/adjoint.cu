// adjoint.cu -- gradients of CCD-plane positions with respect to scheme
// parameters: forward with checkpoints, reverse sweep over surfaces,
// forward-mode sensitivities, and the spot merit's per-ray seeds.
//
// Forward (adjoint_rev.cuh): the fused FP64 engine's per-ray loop (the same
// bits), storing each ray's state at the input of every surface; compiled
// for the scheme's structure like the backward.
//
// Backward (adjoint_rev.cuh): per ray, surfaces last to first, each surface
// recomputed from its checkpoint and its adjoint carried back through its
// stages in one reverse sweep (ray_rev.cuh); the kernel compiled for the
// scheme's structure when NVRTC is there (jit.cpp, rtb_adj_reverse_scheme;
// RTB_SPECIALIZE=0 keeps the generic k_adj_reverse), its sums reproducible.
//
// The same gradient by forward-mode passes (k_adj_backward, selected with
// RTB_ADJOINT_BACKWARD=passes): for surface k the local Jacobian of its
// output state with respect to its input state and to the parameters that
// live on it is recomputed from checkpoint k with dual numbers, W directions
// per pass, and contracted with the output adjoint.  The surface's
// dual-number constants of every pass (which do not depend on the ray) are
// built once per call into a table (k_build_surfd) that all threads read.
//
// Translation unit compiled with --fmad=false: the dual numbers' values are
// the plain engine's.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "engine.cuh"
#include "adjoint_rev.cuh"
#include "jit.h"
#include "ray_ad.cuh"
#include "trace_common.cuh"

namespace rtb {

namespace {

// directions per dual pass of the backward sweep: each pass recomputes the
// surface's values (with their IEEE divisions) once for kAdjW tangents; on
// C4 (1e7 rays, 24 parameters) 2, 3, 4, 6, 8 ran 53, 42, 42, 50, 59 ms
constexpr int kAdjW = 4;
constexpr int kMeritThreads = 256;
constexpr int kMeritParts = 32;    // fixed split of each group's rays (deterministic sums)

// The forward through any scheme (adjoint_rev.cuh).
__global__ void __launch_bounds__(256) k_adj_forward(AdjArgs a, DevRays in, unsigned long long* counts,
                                                     unsigned* err) {
    adj_forward<RtAdjForward>(a, in, counts, err);
}

// The dual-number surface constants of pass (k, d0) of the backward sweep:
// lane l differentiates state component d0 + l (< 6) or the surface's
// parameter d0 + l - 6.
// The state directions of surface k's backward passes.  The first surface's
// input is the entrance ray, which no parameter moves: none.  A later
// surface's input is the previous surface's output, whose cosines form a unit
// vector: every perturbation of them lies in the plane orthogonal to the
// direction, so the input adjoint is needed only there -- the three position
// components and two tangent directions of the cosines, 5 instead of 6.
__host__ __device__ __forceinline__ int backward_state_dirs(int k) { return k == 0 ? 0 : 5; }

// Direction d of a pass: state seed 0..2 (X, Y, Z), 6 or 7 (the cosines'
// tangent directions), or parameter d - n_state of the surface.
__device__ __forceinline__ void backward_seeds(const AdjArgs& a, int k, int d0, ad::Seeds<kAdjW>& sd) {
    const int ns = backward_state_dirs(k);
    const int ndir = ns + a.surf_nparams[k];
    sd.dense = nullptr;
    for (int l = 0; l < kAdjW; ++l) {
        const int d = d0 + l;
        sd.state[l] = (d < ns) ? (d < 3 ? d : 6 + (d - 3)) : -1;
        sd.param[l] = (d >= ns && d < ndir) ? a.surf_params[k * RTB_ADJ_MAX_PARAMS + (d - ns)] : -1;
    }
}

// An orthonormal pair spanning the plane orthogonal to the unit vector c:
// t1 = c x e / |c x e| with e the axis least aligned with c, t2 = c x t1.
__device__ __forceinline__ void tangent_pair(const double c[3], double t1[3], double t2[3]) {
    const double ax = fabs(c[0]), ay = fabs(c[1]), az = fabs(c[2]);
    if (ax <= ay && ax <= az) {
        t1[0] = 0.0; t1[1] = c[2]; t1[2] = -c[1];
    } else if (ay <= az) {
        t1[0] = -c[2]; t1[1] = 0.0; t1[2] = c[0];
    } else {
        t1[0] = c[1]; t1[1] = -c[0]; t1[2] = 0.0;
    }
    const double inv = 1.0 / sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    t1[0] *= inv; t1[1] *= inv; t1[2] *= inv;
    t2[0] = c[1] * t1[2] - c[2] * t1[1];
    t2[1] = c[2] * t1[0] - c[0] * t1[2];
    t2[2] = c[0] * t1[1] - c[1] * t1[0];
}

// One thread per table entry (k, d0).
__global__ void k_build_surfd(AdjArgs a, const int2* entries, int n_entries, ad::SurfD<kAdjW>* table) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_entries) return;
    const int k = entries[e].x;
    ad::Seeds<kAdjW> sd;
    backward_seeds(a, k, entries[e].y, sd);
    ad::make_surfd(a.sch->s[k], k, a.map, a.n_params, sd, table[e]);
}

// The forward-mode constants of surface k along the direction dtheta.
__global__ void k_build_surfd_dense(AdjArgs a, const double* dtheta, ad::SurfD<1>* table) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.sch->n_surfaces) return;
    ad::Seeds<1> sd;
    sd.dense = dtheta;
    sd.state[0] = -1;
    sd.param[0] = -1;
    ad::make_surfd(a.sch->s[k], k, a.map, a.n_params, sd, table[k]);
}

// Rays are taken 32 at a time per warp, every lane of a warp the same number
// of steps, so the warp can sum each parameter's contributions with shuffles.
// first_entry[k]: the table entry of surface k's first pass.  Four blocks per
// SM (at most 128 registers): 217 ms on C4's 1e7 rays against 259 ms at the
// 168 registers the compiler takes unbounded and 256 ms at six blocks.
__global__ void __launch_bounds__(kAdjThreads, 4) k_adj_backward(AdjArgs a, const ad::SurfD<kAdjW>* table,
                                                              const int* first_entry, const double* gX,
                                                              const double* gY, double* partial) {
    __shared__ double acc[kAdjWarps][RTB_ADJ_MAX_PARAMS];
    const DevScheme* sch = a.sch;
    const int ns = sch->n_surfaces;
    const int P = a.n_params;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int p = lane; p < P; p += 32) acc[warp][p] = 0.0;
    __syncwarp();
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x + (size_t)warp * 32; i0 < a.n; i0 += gstride()) {
        const size_t i = i0 + lane;
        bool act = i < a.n && a.flag[i] == 1;
        double adj[6] = {act ? gX[i] : 0.0, act ? gY[i] : 0.0, 0.0, 0.0, 0.0, 0.0};
        act = act && !(adj[0] == 0.0 && adj[1] == 0.0);
        if (!__any_sync(0xffffffffu, act)) continue;
        const double lam = act ? a.lambda[i] : 0.0;
        const int b = act ? beam_of(a.beams, a.n_beams, i) : 0;
        for (int k = ns - 1; k >= 0; --k) {
            const DevSurface& s = sch->s[k];
            double st[6];
            if (act)
                for (int c = 0; c < 6; ++c) st[c] = a.ckpt[((size_t)k * 6 + c) * a.n + i];
            const int nst = backward_state_dirs(k);
            const int ndir = nst + a.surf_nparams[k];
            double t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
            if (act && nst) tangent_pair(st + 3, t1, t2);
            double adj_in[6] = {0, 0, 0, 0, 0, 0}, a_t1 = 0.0, a_t2 = 0.0;
            for (int d0 = 0, e = first_entry[k]; d0 < ndir; d0 += kAdjW, ++e) {
                ad::Seeds<kAdjW> sd;
                backward_seeds(a, k, d0, sd);
                ad::RayD<kAdjW> r;
                if (act) {
                    ad::load_state(st, sd, r, t1, t2);
                    ad::surface_step(s, table[e], sch->fixes, a.knots, adj_order(s, a.beams, b), lam, r);
                }
                // the last surface's output is the CCD-plane point: only X, Y
                // carry adjoints.  Components are picked with selects (run-time
                // indices would keep the ray and the adjoints in local memory).
#pragma unroll
                for (int l = 0; l < kAdjW; ++l) {
                    const int d = d0 + l;
                    if (d >= ndir) break;
                    double v = 0.0;
                    if (act) {
                        v += adj[0] * r.X.d[l];
                        v += adj[1] * r.Y.d[l];
                        v += adj[2] * r.Z.d[l];
                        v += adj[3] * r.cX.d[l];
                        v += adj[4] * r.cY.d[l];
                        v += adj[5] * r.cZ.d[l];
                    }
                    if (d < nst) {
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            if (d == c) adj_in[c] = v;
                        if (d == 3) a_t1 = v;
                        if (d == 4) a_t2 = v;
                    } else {
                        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                        if (lane == 0) acc[warp][sd.param[l]] += v;
                    }
                }
            }
            // the cosines' adjoint, in the plane of their perturbations
            for (int c = 0; c < 3; ++c) adj_in[3 + c] = a_t1 * t1[c] + a_t2 * t2[c];
            for (int c = 0; c < 6; ++c) adj[c] = adj_in[c];
        }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        double sum = 0.0;
        for (int w = 0; w < kAdjWarps; ++w) sum += acc[w][p];
        partial[(size_t)blockIdx.x * P + p] = sum;
    }
}

// The reverse sweep of any scheme (adjoint_rev.cuh).
__global__ void __launch_bounds__(kAdjThreads, 4) k_adj_reverse(AdjArgs a, const double* gX, const double* gY,
                                                             double* partial) {
    adj_reverse<RtAdjSurfaces>(a, gX, gY, partial);
}

// RTB_ADJOINT_BACKWARD=passes: the backward by forward-mode passes.
bool backward_by_passes() {
    const char* e = std::getenv("RTB_ADJOINT_BACKWARD");
    return e && std::strcmp(e, "passes") == 0;
}

__global__ void k_adj_sum_partials(const double* partial, int n_blocks, int P, double* grad) {
    const int p = threadIdx.x;
    if (p >= P) return;
    double s = 0.0;
    for (int b = 0; b < n_blocks; ++b) s += partial[(size_t)b * P + p];
    grad[p] = s;
}

// Forward-mode sensitivities along one parameter direction, through the whole
// scheme from checkpoint 0 (the input rays); table[k]: surface k's constants
// along that direction.
__global__ void __launch_bounds__(kAdjThreads) k_adj_jvp(AdjArgs a, const ad::SurfD<1>* table, double* dX,
                                                         double* dY) {
    adj_jvp<RtAdjJvp>(a, table, dX, dY);
}

// One wavelength group of the spot merit: rays first + m * stride, m < count.
struct Group {
    uint64_t first, stride, count;
};

// pass 0: count, sum X, sum Y; pass 1: the second moments about the
// centroid, sum dX^2, sum dY^2, sum dX dY.  Block (g, part) sums a fixed
// slice of group g.  The groups of a
// composite beam interleave (group j holds rays j, j + n_lambda, ...), so the
// blocks of all groups for one slice -- launched together, group index
// fastest -- read the same stretch of the arrays, and a sector fetched for
// one group is found in L2 by the others.
__global__ void __launch_bounds__(kMeritThreads) k_group_moments(const Group* groups, const char* flag, const double* X,
                                                                 const double* Y, const double* centroid, int pass,
                                                                 double* partial) {
    const int g = blockIdx.x, part = blockIdx.y;
    const Group G = groups[g];
    const uint64_t per = (G.count + kMeritParts - 1) / kMeritParts;
    const uint64_t m0 = (uint64_t)part * per, m1 = (m0 + per < G.count) ? m0 + per : G.count;
    double v[3] = {0, 0, 0};
    const double cx = pass ? centroid[2 * g] : 0.0, cy = pass ? centroid[2 * g + 1] : 0.0;
    for (uint64_t m = m0 + threadIdx.x; m < m1; m += blockDim.x) {
        const uint64_t i = G.first + m * G.stride;
        if (flag[i] != 1) continue;
        if (pass == 0) {
            v[0] += 1.0;
            v[1] += X[i];
            v[2] += Y[i];
        } else {
            const double dx = X[i] - cx, dy = Y[i] - cy;
            v[0] += dx * dx;
            v[1] += dy * dy;
            v[2] += dx * dy;
        }
    }
    __shared__ double red[3][kMeritThreads];
    for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = v[c];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c) partial[((size_t)g * kMeritParts + part) * 3 + c] = red[c][0];
}

// Seeds of a merit that depends on each group's centroid and second
// moments: for a good ray of group g, with (dX, dY) its offset from the
// centroid (cx, cy), gX = axx dX + axy dY + bx and gY = ayx dX + ayy dY + by;
// coef holds (axx, axy, ayx, ayy, bx, by, cx, cy) per group.  Block (g, part),
// group index fastest, as in k_group_moments.
constexpr int kSeedCoef = 8;

__device__ __forceinline__ void seed_of(const double* k, double x, double y, double& gx, double& gy) {
    const double dx = x - k[6], dy = y - k[7];
    gx = fma(k[0], dx, fma(k[1], dy, k[4]));
    gy = fma(k[2], dx, fma(k[3], dy, k[5]));
}

__global__ void k_group_seeds(const Group* groups, int n_groups, const double* coef, const char* flag, const double* X,
                              const double* Y, double* gX, double* gY) {
    const int g = blockIdx.x;
    if (g >= n_groups) return;
    const Group G = groups[g];
    double k[kSeedCoef];
    for (int j = 0; j < kSeedCoef; ++j) k[j] = coef[kSeedCoef * g + j];
    for (uint64_t m = (uint64_t)blockIdx.y * blockDim.x + threadIdx.x; m < G.count; m += (uint64_t)gridDim.y * blockDim.x) {
        const uint64_t i = G.first + m * G.stride;
        if (flag[i] == 1) {
            seed_of(k, X[i], Y[i], gX[i], gY[i]);
        } else {
            gX[i] = 0.0;
            gY[i] = 0.0;
        }
    }
}

// The same moments and seeds read in index order, for beams of at most
// kMeritThreads wavelengths (composite beams: ray first + j holds wavelength
// j mod n_lambda).  Block c of a beam covers rays [start, end) of it, start a
// multiple of the beam's width E = n_lambda * floor(kMeritThreads /
// n_lambda) past its first ray; thread t < E takes rays start + t, start + t
// + E, ..., all of one wavelength (t mod n_lambda), so the loads and stores
// of a warp are consecutive and each thread keeps its group's sums in
// registers.  The sums stay deterministic: each thread adds its rays in
// order, the threads of a group are added in order, and k_dense_finish adds
// the blocks of a beam in order.
struct DenseBlock {
    uint64_t start, end;  // rays of this block
    int32_t nl, width;    // wavelengths of the beam, threads in use (E)
    int32_t gbase;        // group of the beam's first wavelength
    int32_t pbase;        // first partial of this block: (its index in the beam's blocks) * nl + the beam's offset
};

__global__ void __launch_bounds__(kMeritThreads) k_dense_moments(const DenseBlock* blocks, const char* flag,
                                                                 const double* X, const double* Y,
                                                                 const double* centroid, int pass, double* partial) {
    const DenseBlock B = blocks[blockIdx.x];
    const int t = threadIdx.x;
    double v[3] = {0, 0, 0};
    if (t < B.width) {
        const int g = B.gbase + t % B.nl;
        const double cx = pass ? centroid[2 * g] : 0.0, cy = pass ? centroid[2 * g + 1] : 0.0;
        for (uint64_t i = B.start + t; i < B.end; i += B.width) {
            if (flag[i] != 1) continue;
            if (pass == 0) {
                v[0] += 1.0;
                v[1] += X[i];
                v[2] += Y[i];
            } else {
                const double dx = X[i] - cx, dy = Y[i] - cy;
                v[0] += dx * dx;
                v[1] += dy * dy;
                v[2] += dx * dy;
            }
        }
    }
    __shared__ double red[3][kMeritThreads];
    for (int c = 0; c < 3; ++c) red[c][t] = v[c];
    __syncthreads();
    if (t < B.nl) {
        double w[3] = {0, 0, 0};
        for (int m = t; m < B.width; m += B.nl)
            for (int c = 0; c < 3; ++c) w[c] += red[c][m];
        for (int c = 0; c < 3; ++c) partial[((size_t)B.pbase + t) * 3 + c] = w[c];
    }
}

// Per group (one block each): the partials of its beam's blocks, thread t
// adding blocks t, t + kMeritThreads, ... in order, then the threads' sums by
// a fixed tree.  pass 0 leaves count and centroid in out[6g .. 6g+2] and the
// centroid in `centroid`; pass 1 the second moments in out[6g+3 .. 6g+5].
struct DenseGroup {
    int32_t pbase, nl, n_blocks, lg;  // the beam's first partial, wavelengths, blocks; this group's wavelength
};

__global__ void __launch_bounds__(kMeritThreads) k_dense_finish(const DenseGroup* groups, const double* partial,
                                                                int pass, double* centroid, double* out) {
    const int g = blockIdx.x;
    const DenseGroup G = groups[g];
    double v[3] = {0, 0, 0};
    for (int c = threadIdx.x; c < G.n_blocks; c += blockDim.x)
        for (int k = 0; k < 3; ++k) v[k] += partial[((size_t)G.pbase + (size_t)c * G.nl + G.lg) * 3 + k];
    __shared__ double red[3][kMeritThreads];
    for (int k = 0; k < 3; ++k) red[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    for (int k = 0; k < 3; ++k) v[k] = red[k][0];
    if (pass == 0) {
        out[6 * g] = v[0];
        centroid[2 * g] = out[6 * g + 1] = v[0] > 0 ? v[1] / v[0] : 0.0;
        centroid[2 * g + 1] = out[6 * g + 2] = v[0] > 0 ? v[2] / v[0] : 0.0;
    } else {
        for (int k = 0; k < 3; ++k) out[6 * g + 3 + k] = v[k];
    }
}

__global__ void __launch_bounds__(kMeritThreads) k_dense_seeds(const DenseBlock* blocks, const double* coef,
                                                               const char* flag, const double* X, const double* Y,
                                                               double* gX, double* gY) {
    const DenseBlock B = blocks[blockIdx.x];
    const int t = threadIdx.x;
    if (t >= B.width) return;
    const int g = B.gbase + t % B.nl;
    double k[kSeedCoef];
    for (int j = 0; j < kSeedCoef; ++j) k[j] = coef[kSeedCoef * g + j];
    for (uint64_t i = B.start + t; i < B.end; i += B.width) {
        if (flag[i] == 1) {
            seed_of(k, X[i], Y[i], gX[i], gY[i]);
        } else {
            gX[i] = 0.0;
            gY[i] = 0.0;
        }
    }
}

}  // namespace

}  // namespace rtb

using namespace rtb;

struct rtb_adjoint {
    int device = 0;
    std::vector<rtb_surface> surf;                 // the scheme, tables repointed to...
    std::vector<std::vector<double>> tables;       // ...these copies
    std::vector<rtb_param> params;
    std::vector<int> surf_nparams;                 // parameters per surface
    std::vector<DevBeam> beams_h;
    std::vector<rtb_beam> beams_in;
    uint64_t n = 0;
    uint32_t fixes = 0;
    PreparedScheme ps;
    bool have_forward = false;
    const void* fwd_kernel = nullptr;              // the forward, the reverse sweep and the
    const void* rev_kernel = nullptr;              // sensitivities compiled for the scheme's
    const void* jvp_kernel = nullptr;              // structure, or NULL
    // device
    void* mem = nullptr;
    DevScheme* d_sch = nullptr;
    double* d_knots = nullptr;
    size_t knots_cap = 0;
    DevBeam* d_beams = nullptr;
    ad::ParamRef* d_map = nullptr;
    int* d_surf_params = nullptr;
    int* d_surf_nparams = nullptr;
    double* d_ckpt = nullptr;
    double* d_lambda = nullptr;
    char* d_flag = nullptr;
    double* d_X = nullptr;
    double* d_Y = nullptr;
    unsigned long long* d_counts = nullptr;
    unsigned* d_err = nullptr;
    double* d_grad = nullptr;
    double* d_dtheta = nullptr;
    cudaStream_t stream = nullptr;
};

namespace {

int check_param(const rtb_surface& s, const rtb_param& p) {
    const bool conic = s.cls == RTB_CONIC, toric = s.cls == RTB_TORIC;
    const int N = (s.cls == RTB_PLANE || s.cls == RTB_AUX_CLASS) ? 0 : (int)s.params[2];
    switch (p.kind) {
        case RTB_PARAM_CURVATURE:  // c = 0 switches a conic to the plane / polynomial algorithm
            return ((conic || toric) && s.params[0] != 0.0) ? RTB_OK : RTB_BAD_VALUE;
        case RTB_PARAM_CONIC:      // k = -1 selects the paraboloid's linear root
            return ((conic && s.params[1] != -1.0) || toric) ? RTB_OK : RTB_BAD_VALUE;
        case RTB_PARAM_POLY:
            return ((conic || toric) && p.index >= 0 && p.index < N) ? RTB_OK : RTB_BAD_VALUE;
        case RTB_PARAM_TORIC_CR:
            return toric ? RTB_OK : RTB_BAD_VALUE;
        case RTB_PARAM_DISTANCE:
        case RTB_PARAM_ANGLE:
            return (p.index >= 0 && p.index < 3) ? RTB_OK : RTB_BAD_VALUE;
        case RTB_PARAM_GROOVE_DENSITY:
            return (s.type == RTB_GRATING && s.gr_const > 0.0) ? RTB_OK : RTB_BAD_VALUE;
        default:
            return RTB_BAD_VALUE;
    }
}

double get_param(const rtb_surface& s, const rtb_param& p) {
    switch (p.kind) {
        case RTB_PARAM_CURVATURE: return s.params[0];
        case RTB_PARAM_CONIC: return s.params[1];
        case RTB_PARAM_POLY: return s.params[3 + p.index];
        case RTB_PARAM_TORIC_CR: return s.params[3 + (int)s.params[2]];
        case RTB_PARAM_DISTANCE: return s.distance[p.index];
        case RTB_PARAM_ANGLE: return s.angles_deg[p.index];
        case RTB_PARAM_GROOVE_DENSITY: return 1000.0 / s.gr_const;
        default: return 0.0;
    }
}

void set_param(rtb_surface& s, const rtb_param& p, double v) {
    switch (p.kind) {
        case RTB_PARAM_CURVATURE: s.params[0] = v; break;
        case RTB_PARAM_CONIC: s.params[1] = v; break;
        case RTB_PARAM_POLY: s.params[3 + p.index] = v; break;
        case RTB_PARAM_TORIC_CR: s.params[3 + (int)s.params[2]] = v; break;
        case RTB_PARAM_DISTANCE: s.distance[p.index] = v; break;
        case RTB_PARAM_ANGLE: s.angles_deg[p.index] = v; break;
        case RTB_PARAM_GROOVE_DENSITY: s.gr_const = 1000.0 / v; break;
        default: break;
    }
}

void copy_table(rtb_table& t, std::vector<std::vector<double>>& store) {
    if (t.n == 0 || !t.y) return;
    std::vector<double> v;
    const size_t n = t.n;
    if (n == 1) {
        v.assign(t.y, t.y + 1);
        store.push_back(v);
        t.y = store.back().data();
        t.x = nullptr;
        t.y2 = nullptr;
        return;
    }
    v.resize(3 * n);
    std::memcpy(v.data(), t.x, n * sizeof(double));
    std::memcpy(v.data() + n, t.y, n * sizeof(double));
    if (t.y2) std::memcpy(v.data() + 2 * n, t.y2, n * sizeof(double));
    store.push_back(std::move(v));
    const double* b = store.back().data();
    t.x = b;
    t.y = b + n;
    t.y2 = t.y2 ? b + 2 * n : nullptr;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

unsigned adj_grid(uint64_t n, int threads) {
    size_t blocks = (n + threads - 1) / threads;
    const size_t cap = (size_t)engine().sm_count * 8;
    if (blocks > cap) blocks = cap;
    return (unsigned)(blocks ? blocks : 1);
}

AdjArgs adj_args(const rtb_adjoint* c) {
    AdjArgs a;
    a.sch = c->d_sch;
    a.knots = c->d_knots;
    a.beams = c->d_beams;
    a.n_beams = (int)c->beams_h.size();
    a.map = c->d_map;
    a.n_params = (int)c->params.size();
    a.surf_params = c->d_surf_params;
    a.surf_nparams = c->d_surf_nparams;
    a.ckpt = c->d_ckpt;
    a.lambda = c->d_lambda;
    a.flag = c->d_flag;
    a.X = c->d_X;
    a.Y = c->d_Y;
    a.n = c->n;
    return a;
}

}  // namespace

extern "C" {

int rtb_adjoint_create(const rtb_surface* surfaces, size_t n_surfaces, const rtb_param* params, size_t n_params,
                       const rtb_beam* beams, size_t n_beams, uint64_t n_rays, uint32_t fixes, rtb_adjoint** out) {
    if (!out || !surfaces || n_surfaces == 0 || n_surfaces > RTB_MAX_SURFACES || !beams || n_beams == 0 ||
        n_rays == 0 || (n_params && !params) || n_params > RTB_ADJ_MAX_PARAMS)
        return RTB_BAD_VALUE;
    *out = nullptr;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    rtb_adjoint* c = new rtb_adjoint();
    cudaGetDevice(&c->device);
    c->surf.assign(surfaces, surfaces + n_surfaces);
    c->tables.reserve(2 * n_surfaces);
    for (auto& s : c->surf) {
        copy_table(s.n1, c->tables);
        copy_table(s.n2, c->tables);
    }
    c->params.assign(params, params + n_params);
    for (const auto& p : c->params) {
        if (p.surface < 0 || p.surface >= (int)n_surfaces || check_param(c->surf[p.surface], p) != RTB_OK) {
            delete c;
            return RTB_BAD_VALUE;
        }
    }
    c->n = n_rays;
    c->fixes = fixes;
    c->beams_in.assign(beams, beams + n_beams);
    if ((st = check_beams(beams, n_beams, n_rays, c->beams_h)) != RTB_OK ||
        (st = prepare_scheme(c->surf.data(), n_surfaces, fixes, 0, c->ps)) != RTB_OK) {
        delete c;
        return st;
    }
    // parameter lists per surface
    std::vector<int> sp(n_surfaces * RTB_ADJ_MAX_PARAMS, -1), sn(n_surfaces, 0);
    std::vector<ad::ParamRef> map(n_params ? n_params : 1);
    for (size_t j = 0; j < n_params; ++j) {
        const rtb_param& p = c->params[j];
        map[j] = ad::ParamRef{p.surface, p.kind, p.index, 0};
        sp[p.surface * RTB_ADJ_MAX_PARAMS + sn[p.surface]++] = (int)j;
    }
    c->surf_nparams = sn;
    // one allocation: scheme, knots (room for the largest table set), beams,
    // map, lists, counters, grad; then the per-ray arrays
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    c->knots_cap = c->ps.knots.size();
    const size_t ns1 = 3 * n_surfaces + 1;
    size_t off = 0;
    const size_t o_sch = off; off += al(sizeof(DevScheme));
    const size_t o_kn = off; off += al(c->knots_cap * sizeof(double));
    const size_t o_bm = off; off += al(n_beams * sizeof(DevBeam));
    const size_t o_map = off; off += al(map.size() * sizeof(ad::ParamRef));
    const size_t o_sp = off; off += al(sp.size() * sizeof(int));
    const size_t o_sn = off; off += al(sn.size() * sizeof(int));
    const size_t o_cnt = off; off += al(n_beams * ns1 * 8);
    const size_t o_err = off; off += 256;
    const size_t o_grad = off; off += al(RTB_ADJ_MAX_PARAMS * sizeof(double));
    const size_t o_dth = off; off += al(RTB_ADJ_MAX_PARAMS * sizeof(double));
    const size_t o_ck = off; off += al(n_rays * 6 * n_surfaces * sizeof(double));
    const size_t o_lam = off; off += al(n_rays * sizeof(double));
    const size_t o_x = off; off += al(n_rays * sizeof(double));
    const size_t o_y = off; off += al(n_rays * sizeof(double));
    const size_t o_fl = off; off += al(n_rays);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = dev_malloc((void**)&c->mem, off);
    if (e != cudaSuccess) {
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return cuda_status(e);
    }
    char* b = static_cast<char*>(c->mem);
    c->d_sch = reinterpret_cast<DevScheme*>(b + o_sch);
    c->d_knots = reinterpret_cast<double*>(b + o_kn);
    c->d_beams = reinterpret_cast<DevBeam*>(b + o_bm);
    c->d_map = reinterpret_cast<ad::ParamRef*>(b + o_map);
    c->d_surf_params = reinterpret_cast<int*>(b + o_sp);
    c->d_surf_nparams = reinterpret_cast<int*>(b + o_sn);
    c->d_counts = reinterpret_cast<unsigned long long*>(b + o_cnt);
    c->d_err = reinterpret_cast<unsigned*>(b + o_err);
    c->d_grad = reinterpret_cast<double*>(b + o_grad);
    c->d_dtheta = reinterpret_cast<double*>(b + o_dth);
    c->d_ckpt = reinterpret_cast<double*>(b + o_ck);
    c->d_lambda = reinterpret_cast<double*>(b + o_lam);
    c->d_X = reinterpret_cast<double*>(b + o_x);
    c->d_Y = reinterpret_cast<double*>(b + o_y);
    c->d_flag = b + o_fl;
    e = cudaMemcpyAsync(c->d_beams, c->beams_h.data(), n_beams * sizeof(DevBeam), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d_map, map.data(), map.size() * sizeof(ad::ParamRef), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d_surf_params, sp.data(), sp.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d_surf_nparams, sn.data(), sn.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaFree(c->mem);
        cudaStreamDestroy(c->stream);
        delete c;
        return cuda_status(e);
    }
    // the reverse sweep compiled for the scheme's structure, which the
    // parameters cannot change (check_param; rtb_adjoint_forward checks the
    // intersection kinds); the generic kernel when NVRTC is unavailable
    if (specialize_enabled()) {
        std::string why;
        const void *f = nullptr, *r = nullptr, *j = nullptr;
        if (adjoint_kernels(c->ps.sch, &f, &r, &j, &why) == RTB_OK) {
            c->fwd_kernel = f;
            c->rev_kernel = r;
            c->jvp_kernel = j;
        }
    }
    *out = c;
    return RTB_OK;
}

int rtb_adjoint_theta(const rtb_adjoint* c, double* theta) {
    if (!c || (!theta && !c->params.empty())) return RTB_BAD_VALUE;
    for (size_t j = 0; j < c->params.size(); ++j) theta[j] = get_param(c->surf[c->params[j].surface], c->params[j]);
    return RTB_OK;
}

int rtb_adjoint_forward(rtb_adjoint* c, const double* theta, const rtb_rays* rays, double* X, double* Y, char* flag,
                        rtb_trace_stats* stats, void* stream) {
    Range range("rtb_adjoint_forward");
    if (!c || !rays || rays->n != c->n || !rays->flag) return RTB_BAD_VALUE;
    DeviceGuard dg(c->device);
    Lock l;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    std::vector<rtb_surface> sf = c->surf;
    if (theta)
        for (size_t j = 0; j < c->params.size(); ++j) {
            if (c->params[j].kind == RTB_PARAM_GROOVE_DENSITY && !(theta[j] > 0.0)) return RTB_BAD_VALUE;
            set_param(sf[c->params[j].surface], c->params[j], theta[j]);
        }
    PreparedScheme ps;
    int st = prepare_scheme(sf.data(), sf.size(), c->fixes, 0, ps);
    if (st != RTB_OK) return st;
    // a parameter must not switch a surface's algorithm (check_param at create)
    for (size_t k = 0; k < sf.size(); ++k)
        if (ps.sch.s[k].kind != c->ps.sch.s[k].kind) return RTB_BAD_VALUE;
    if (ps.knots.size() > c->knots_cap) return RTB_BAD_VALUE;
    c->ps = ps;
    const size_t ns1 = 3 * sf.size() + 1;
    const size_t nb = c->beams_h.size();
    RTB_CUDA_TRY(cudaMemcpyAsync(c->d_sch, &ps.sch, sizeof(DevScheme), cudaMemcpyHostToDevice, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(c->d_knots, ps.knots.data(), ps.knots.size() * sizeof(double), cudaMemcpyHostToDevice,
                                 s));
    RTB_CUDA_TRY(cudaMemsetAsync(c->d_counts, 0, nb * ns1 * 8, s));
    RTB_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, 4, s));
    AdjArgs a = adj_args(c);
    DevRays in = dev_rays(rays);
    if (c->fwd_kernel) {
        unsigned long long* counts = c->d_counts;
        unsigned* err = c->d_err;
        void* args[] = {&a, &in, &counts, &err};
        RTB_CUDA_TRY(cudaLaunchKernel(c->fwd_kernel, dim3(adj_grid(c->n, 256)), dim3(256), args, 0, s));
    } else {
        k_adj_forward<<<adj_grid(c->n, 256), 256, 0, s>>>(a, in, c->d_counts, c->d_err);
    }
    RTB_CUDA_TRY(cudaGetLastError());
    if (X) RTB_CUDA_TRY(cudaMemcpyAsync(X, c->d_X, c->n * 8, cudaMemcpyDeviceToDevice, s));
    if (Y) RTB_CUDA_TRY(cudaMemcpyAsync(Y, c->d_Y, c->n * 8, cudaMemcpyDeviceToDevice, s));
    if (flag) RTB_CUDA_TRY(cudaMemcpyAsync(flag, c->d_flag, c->n, cudaMemcpyDeviceToDevice, s));
    std::vector<unsigned long long> counts(nb * ns1);
    unsigned err = 0;
    RTB_CUDA_TRY(cudaMemcpyAsync(counts.data(), c->d_counts, counts.size() * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(&err, c->d_err, 4, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    c->have_forward = true;
    return trace_result(ps, counts.data(), err, (int)nb, stats);
}

int rtb_adjoint_backward(rtb_adjoint* c, const double* gX, const double* gY, double* grad, void* stream) {
    Range range("rtb_adjoint_backward");
    if (!c || !gX || !gY || (!grad && !c->params.empty()) || !c->have_forward) return RTB_BAD_VALUE;
    if (c->params.empty()) return RTB_OK;
    DeviceGuard dg(c->device);
    Lock l;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    const int P = (int)c->params.size();
    const unsigned grid = adj_grid(c->n, kAdjThreads);
    AdjArgs a = adj_args(c);
    if (!backward_by_passes()) {
        DevBuf part;
        int st = part.alloc((size_t)grid * P * sizeof(double), s);
        if (st != RTB_OK) return st;
        double* partial = part.as<double>();
        if (c->rev_kernel) {
            void* args[] = {&a, &gX, &gY, &partial};
            RTB_CUDA_TRY(cudaLaunchKernel(c->rev_kernel, dim3(grid), dim3(kAdjThreads), args, 0, s));
        } else {
            k_adj_reverse<<<grid, kAdjThreads, 0, s>>>(a, gX, gY, partial);
        }
        RTB_CUDA_TRY(cudaGetLastError());
        k_adj_sum_partials<<<1, RTB_ADJ_MAX_PARAMS, 0, s>>>(part.as<double>(), (int)grid, P, c->d_grad);
        RTB_CUDA_TRY(cudaGetLastError());
        RTB_CUDA_TRY(cudaMemcpyAsync(grad, c->d_grad, P * sizeof(double), cudaMemcpyDeviceToHost, s));
        RTB_CUDA_TRY(cudaStreamSynchronize(s));
        return RTB_OK;
    }
    // the passes of every surface: (k, first direction)
    std::vector<int2> entries;
    std::vector<int> first(c->surf_nparams.size());
    for (size_t k = 0; k < c->surf_nparams.size(); ++k) {
        first[k] = (int)entries.size();
        for (int d0 = 0; d0 < backward_state_dirs((int)k) + c->surf_nparams[k]; d0 += kAdjW)
            entries.push_back(make_int2((int)k, d0));
    }
    const size_t ne = entries.size();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t o_ent = al(ne * sizeof(ad::SurfD<kAdjW>)), o_first = o_ent + al(ne * sizeof(int2)),
                 o_part = o_first + al(first.size() * sizeof(int));
    DevBuf buf;
    int st = buf.alloc(o_part + (size_t)grid * P * sizeof(double), s);
    if (st != RTB_OK) return st;
    char* p = buf.as<char>();
    auto* table = reinterpret_cast<ad::SurfD<kAdjW>*>(p);
    auto* d_ent = reinterpret_cast<int2*>(p + o_ent);
    auto* d_first = reinterpret_cast<int*>(p + o_first);
    double* partial = reinterpret_cast<double*>(p + o_part);
    RTB_CUDA_TRY(cudaMemcpyAsync(d_ent, entries.data(), ne * sizeof(int2), cudaMemcpyHostToDevice, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    k_build_surfd<<<(unsigned)((ne + 63) / 64), 64, 0, s>>>(a, d_ent, (int)ne, table);
    RTB_CUDA_TRY(cudaGetLastError());
    k_adj_backward<<<grid, kAdjThreads, 0, s>>>(a, table, d_first, gX, gY, partial);
    RTB_CUDA_TRY(cudaGetLastError());
    k_adj_sum_partials<<<1, RTB_ADJ_MAX_PARAMS, 0, s>>>(partial, (int)grid, P, c->d_grad);
    RTB_CUDA_TRY(cudaGetLastError());
    RTB_CUDA_TRY(cudaMemcpyAsync(grad, c->d_grad, P * sizeof(double), cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    return RTB_OK;
}

int rtb_adjoint_jvp(rtb_adjoint* c, const double* dtheta, double* dX, double* dY, void* stream) {
    Range range("rtb_adjoint_jvp");
    if (!c || !dX || !dY || (!dtheta && !c->params.empty()) || !c->have_forward) return RTB_BAD_VALUE;
    DeviceGuard dg(c->device);
    Lock l;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    std::vector<double> d(RTB_ADJ_MAX_PARAMS, 0.0);
    for (size_t j = 0; j < c->params.size(); ++j) d[j] = dtheta[j];
    RTB_CUDA_TRY(cudaMemcpyAsync(c->d_dtheta, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    AdjArgs a = adj_args(c);
    const int ns = (int)c->surf_nparams.size();
    DevBuf table;
    int st = table.alloc((size_t)ns * sizeof(ad::SurfD<1>), s);
    if (st != RTB_OK) return st;
    k_build_surfd_dense<<<(unsigned)((ns + 31) / 32), 32, 0, s>>>(a, c->d_dtheta, table.as<ad::SurfD<1>>());
    RTB_CUDA_TRY(cudaGetLastError());
    const ad::SurfD<1>* tab = table.as<ad::SurfD<1>>();
    if (c->jvp_kernel) {
        void* args[] = {&a, &tab, &dX, &dY};
        RTB_CUDA_TRY(cudaLaunchKernel(c->jvp_kernel, dim3(adj_grid(c->n, kAdjThreads)), dim3(kAdjThreads), args, 0, s));
    } else {
        k_adj_jvp<<<adj_grid(c->n, kAdjThreads), kAdjThreads, 0, s>>>(a, tab, dX, dY);
    }
    RTB_CUDA_TRY(cudaGetLastError());
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    return RTB_OK;
}

}  // extern "C"

namespace {

// The moments of every wavelength group of the last forward (group g = beam
// b, wavelength index j; rays first_ray + j + m * n_lambda, good rays only)
// and the kernels that turn per-group seed coefficients into per-ray seeds.
struct GroupMoments {
    std::vector<double> n, cx, cy, sxx, syy, sxy;  // count, centroid, second moments about it
};

class MeritPass {
  public:
    MeritPass(rtb_adjoint* c, cudaStream_t s) : c_(c), s_(s) {}

    int moments(GroupMoments& m) {
        for (const auto& b : c_->beams_in) {
            const uint64_t nl = b.n_lambda ? b.n_lambda : 1;
            for (uint64_t j = 0; j < nl; ++j) {
                const uint64_t cnt = (b.n_rays > j) ? (b.n_rays - j + nl - 1) / nl : 0;
                groups_.push_back(Group{b.first_ray + j, nl, cnt});
            }
        }
        G_ = (int)groups_.size();
        if (G_ == 0 || G_ > 65535) return RTB_BAD_VALUE;
        // index-order (dense) path: every beam of at most kMeritThreads wavelengths
        dense_ = true;
        for (const auto& b : c_->beams_in) dense_ = dense_ && (b.n_lambda ? b.n_lambda : 1) <= (uint64_t)kMeritThreads;
        if (dense_) {
            constexpr uint64_t kRaysPerThread = 8;
            uint64_t pbase = 0;
            int32_t gbase = 0;
            for (const auto& b : c_->beams_in) {
                const int32_t nl = (int32_t)(b.n_lambda ? b.n_lambda : 1);
                const int32_t width = nl * (kMeritThreads / nl);
                const uint64_t chunk = (uint64_t)width * kRaysPerThread;
                const uint64_t nblk = (b.n_rays + chunk - 1) / chunk;
                for (uint64_t k = 0; k < nblk; ++k) {
                    const uint64_t start = b.first_ray + k * chunk;
                    const uint64_t end = std::min(b.first_ray + b.n_rays, start + chunk);
                    dblocks_.push_back(DenseBlock{start, end, nl, width, gbase, (int32_t)(pbase + k * (uint64_t)nl)});
                }
                for (int32_t j = 0; j < nl; ++j) dgroups_.push_back(DenseGroup{(int32_t)pbase, nl, (int32_t)nblk, j});
                pbase += nblk * (uint64_t)nl;
                gbase += nl;
                if (pbase > (uint64_t)INT32_MAX || dblocks_.size() > (size_t)INT32_MAX) dense_ = false;
            }
        }
        const size_t n_part = dense_ ? (size_t)dgroups_.back().pbase + (size_t)dgroups_.back().n_blocks * dgroups_.back().nl
                                     : (size_t)G_ * kMeritParts;
        const size_t tab_bytes = dense_ ? a256(dblocks_.size() * sizeof(DenseBlock)) + a256(G_ * sizeof(DenseGroup))
                                        : a256(G_ * sizeof(Group));
        const size_t part_bytes = a256(n_part * 3 * sizeof(double));
        int st = buf_.alloc(tab_bytes + part_bytes + (size_t)G_ * (kSeedCoef + 2 + 6) * sizeof(double), s_);
        if (st != RTB_OK) return st;
        char* p = buf_.as<char>();
        d_groups_ = reinterpret_cast<Group*>(p);
        d_blocks_ = reinterpret_cast<DenseBlock*>(p);
        DenseGroup* d_dgroups = reinterpret_cast<DenseGroup*>(p + a256(dblocks_.size() * sizeof(DenseBlock)));
        double* d_part = reinterpret_cast<double*>(p + tab_bytes);
        d_coef_ = reinterpret_cast<double*>(p + tab_bytes + part_bytes);  // kSeedCoef G
        double* d_cen = d_coef_ + (size_t)kSeedCoef * G_;                    // 2 G
        double* d_out = d_cen + 2 * (size_t)G_;                              // 6 G
        m.n.assign(G_, 0.0);
        m.cx.assign(G_, 0.0);
        m.cy.assign(G_, 0.0);
        m.sxx.assign(G_, 0.0);
        m.syy.assign(G_, 0.0);
        m.sxy.assign(G_, 0.0);
        cudaStream_t s = s_;
        if (dense_) {
            if (!dblocks_.empty())
                RTB_CUDA_TRY(cudaMemcpyAsync(d_blocks_, dblocks_.data(), dblocks_.size() * sizeof(DenseBlock),
                                             cudaMemcpyHostToDevice, s));
            RTB_CUDA_TRY(cudaMemcpyAsync(d_dgroups, dgroups_.data(), G_ * sizeof(DenseGroup), cudaMemcpyHostToDevice, s));
            for (int pass = 0; pass < 2; ++pass) {
                if (!dblocks_.empty())
                    k_dense_moments<<<(unsigned)dblocks_.size(), kMeritThreads, 0, s>>>(d_blocks_, c_->d_flag, c_->d_X,
                                                                                        c_->d_Y, d_cen, pass, d_part);
                k_dense_finish<<<G_, kMeritThreads, 0, s>>>(d_dgroups, d_part, pass, d_cen, d_out);
                RTB_CUDA_TRY(cudaGetLastError());
            }
            std::vector<double> out(6 * (size_t)G_);
            RTB_CUDA_TRY(cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
            RTB_CUDA_TRY(cudaStreamSynchronize(s));
            for (int g = 0; g < G_; ++g) {
                m.n[g] = out[6 * g];
                m.cx[g] = out[6 * g + 1];
                m.cy[g] = out[6 * g + 2];
                m.sxx[g] = out[6 * g + 3];
                m.syy[g] = out[6 * g + 4];
                m.sxy[g] = out[6 * g + 5];
            }
            return RTB_OK;
        }
        RTB_CUDA_TRY(cudaMemcpyAsync(d_groups_, groups_.data(), G_ * sizeof(Group), cudaMemcpyHostToDevice, s));
        std::vector<double> part((size_t)G_ * kMeritParts * 3), cen(2 * (size_t)G_);
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1)
                RTB_CUDA_TRY(cudaMemcpyAsync(d_cen, cen.data(), cen.size() * sizeof(double), cudaMemcpyHostToDevice, s));
            k_group_moments<<<dim3(G_, kMeritParts), kMeritThreads, 0, s>>>(d_groups_, c_->d_flag, c_->d_X, c_->d_Y,
                                                                           d_cen, pass, d_part);
            RTB_CUDA_TRY(cudaGetLastError());
            RTB_CUDA_TRY(cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
            RTB_CUDA_TRY(cudaStreamSynchronize(s));
            for (int g = 0; g < G_; ++g) {
                double v[3] = {0, 0, 0};
                for (int q = 0; q < kMeritParts; ++q)
                    for (int k = 0; k < 3; ++k) v[k] += part[((size_t)g * kMeritParts + q) * 3 + k];
                if (pass == 0) {
                    m.n[g] = v[0];
                    cen[2 * g] = m.cx[g] = v[0] > 0 ? v[1] / v[0] : 0.0;
                    cen[2 * g + 1] = m.cy[g] = v[0] > 0 ? v[2] / v[0] : 0.0;
                } else {
                    m.sxx[g] = v[0];
                    m.syy[g] = v[1];
                    m.sxy[g] = v[2];
                }
            }
        }
        return RTB_OK;
    }

    // Per-ray seeds from kSeedCoef coefficients per group (see seed_of); rays
    // outside every group get 0.
    int seeds(const std::vector<double>& coef, double* gX, double* gY) {
        cudaStream_t s = s_;
        // rays outside every group: all of them here, or (dense path, which
        // writes every ray of every beam) those between the beams
        uint64_t from = 0;
        auto zero = [&](uint64_t a, uint64_t b) -> cudaError_t {
            if (b <= a) return cudaSuccess;
            cudaError_t e = cudaMemsetAsync(gX + a, 0, (b - a) * sizeof(double), s);
            return e == cudaSuccess ? cudaMemsetAsync(gY + a, 0, (b - a) * sizeof(double), s) : e;
        };
        if (dense_) {
            for (const auto& b : c_->beams_in) {
                RTB_CUDA_TRY(zero(from, b.first_ray));
                from = b.first_ray + b.n_rays;
            }
        }
        RTB_CUDA_TRY(zero(from, c_->n));
        RTB_CUDA_TRY(cudaMemcpyAsync(d_coef_, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        if (dense_) {
            if (!dblocks_.empty())
                k_dense_seeds<<<(unsigned)dblocks_.size(), kMeritThreads, 0, s>>>(d_blocks_, d_coef_, c_->d_flag,
                                                                                  c_->d_X, c_->d_Y, gX, gY);
        } else {
            k_group_seeds<<<dim3(G_, 64), 256, 0, s>>>(d_groups_, G_, d_coef_, c_->d_flag, c_->d_X, c_->d_Y, gX, gY);
        }
        RTB_CUDA_TRY(cudaGetLastError());
        RTB_CUDA_TRY(cudaStreamSynchronize(s));
        return RTB_OK;
    }

    int n_groups() const { return G_; }

  private:
    static size_t a256(size_t b) { return (b + 255) / 256 * 256; }
    rtb_adjoint* c_;
    cudaStream_t s_;
    std::vector<Group> groups_;
    std::vector<DenseBlock> dblocks_;
    std::vector<DenseGroup> dgroups_;
    int G_ = 0;
    bool dense_ = false;
    DevBuf buf_;
    Group* d_groups_ = nullptr;
    DenseBlock* d_blocks_ = nullptr;
    double* d_coef_ = nullptr;
};

}  // namespace

extern "C" {

int rtb_adjoint_spot_merit(rtb_adjoint* c, const double* target_x, double weight, double* merit, double* gX,
                           double* gY, void* stream) {
    Range range("rtb_adjoint_spot_merit");
    if (!c || !target_x || !merit || !c->have_forward || ((gX == nullptr) != (gY == nullptr))) return RTB_BAD_VALUE;
    DeviceGuard dg(c->device);
    Lock l;
    MeritPass mp(c, stream ? (cudaStream_t)stream : c->stream);
    GroupMoments m;
    int st = mp.moments(m);
    if (st != RTB_OK) return st;
    const int G = mp.n_groups();
    double M = 0.0;
    std::vector<double> coef((size_t)kSeedCoef * G, 0.0);
    for (int g = 0; g < G; ++g) {
        if (!(m.n[g] > 0)) continue;
        const double rms = std::sqrt((m.sxx[g] + m.syy[g]) / m.n[g]);
        const double dx = m.cx[g] - target_x[g];
        M += rms + weight * dx * dx;
        double* k = &coef[(size_t)kSeedCoef * g];
        const double a = rms > 0 ? 1.0 / (m.n[g] * rms) : 0.0;  // d rms / dX_i = (X_i - xbar) / (N rms)
        k[0] = k[3] = a;
        k[4] = 2.0 * weight * dx / m.n[g];  // d w (xbar - t)^2 / dX_i
        k[6] = m.cx[g];
        k[7] = m.cy[g];
    }
    *merit = M;
    return gX ? mp.seeds(coef, gX, gY) : RTB_OK;
}

int rtb_adjoint_resolution_merit(rtb_adjoint* c, const double* lambda, double ux, double uy, double* merit,
                                 double* gX, double* gY, void* stream) {
    Range range("rtb_adjoint_resolution_merit");
    if (!c || !lambda || !merit || !c->have_forward || ((gX == nullptr) != (gY == nullptr))) return RTB_BAD_VALUE;
    const double un = std::hypot(ux, uy);
    if (!(un > 0.0) || !std::isfinite(un)) return RTB_BAD_VALUE;
    ux /= un;
    uy /= un;
    DeviceGuard dg(c->device);
    Lock l;
    MeritPass mp(c, stream ? (cudaStream_t)stream : c->stream);
    GroupMoments m;
    int st = mp.moments(m);
    if (st != RTB_OK) return st;
    const int G = mp.n_groups();
    for (int g = 0; g < G; ++g)
        if (!std::isfinite(lambda[g]) || !(lambda[g] > 0.0)) return RTB_BAD_VALUE;
    // along the dispersion direction u: the centroid p_g and RMS width s_g of
    // each group's spot
    std::vector<double> p(G, 0.0), sg(G, 0.0), dM_dp(G, 0.0), dM_ds(G, 0.0);
    for (int g = 0; g < G; ++g) {
        if (!(m.n[g] > 0)) continue;
        p[g] = ux * m.cx[g] + uy * m.cy[g];
        const double v = (ux * ux * m.sxx[g] + 2.0 * ux * uy * m.sxy[g] + uy * uy * m.syy[g]) / m.n[g];
        sg[g] = std::sqrt(std::max(v, 0.0));
    }
    // pairs of neighbouring wavelengths of a beam, both with good rays: the
    // width of a resolution element in wavelength over its mean wavelength,
    // (s_g + s_h) / 2 * |lambda_h - lambda_g| / |p_h - p_g| / ((lambda_g + lambda_h) / 2)
    double M = 0.0;
    int g0 = 0;
    for (const auto& b : c->beams_in) {
        const int nl = (int)(b.n_lambda ? b.n_lambda : 1);
        for (int j = 0; j + 1 < nl; ++j) {
            const int g = g0 + j, h = g + 1;
            if (!(m.n[g] > 0) || !(m.n[h] > 0)) continue;
            const double d = p[h] - p[g];
            if (d == 0.0) return RTB_BAD_VALUE;  // two wavelengths on one spot: no resolution to speak of
            const double w = std::fabs(lambda[h] - lambda[g]) / (0.5 * (lambda[g] + lambda[h]));
            const double ad = std::fabs(d), sbar = 0.5 * (sg[g] + sg[h]);
            M += w * sbar / ad;
            dM_ds[g] += 0.5 * w / ad;
            dM_ds[h] += 0.5 * w / ad;
            const double dd = -w * sbar / (ad * d);  // d(w sbar / |d|) / dd
            dM_dp[h] += dd;
            dM_dp[g] -= dd;
        }
        g0 += nl;
    }
    *merit = M;
    if (!gX) return RTB_OK;
    // d/dq_i of p_g = 1 / N_g, of s_g = (q_i - p_g) / (N_g s_g), q_i = u . (X_i, Y_i):
    // dM/dX_i = ux (dM/dp_g / N_g + dM/ds_g (q_i - p_g) / (N_g s_g)), likewise Y
    std::vector<double> coef((size_t)kSeedCoef * G, 0.0);
    for (int g = 0; g < G; ++g) {
        if (!(m.n[g] > 0)) continue;
        double* k = &coef[(size_t)kSeedCoef * g];
        const double a = sg[g] > 0 ? dM_ds[g] / (m.n[g] * sg[g]) : 0.0, bp = dM_dp[g] / m.n[g];
        k[0] = a * ux * ux;
        k[1] = a * ux * uy;
        k[2] = a * ux * uy;
        k[3] = a * uy * uy;
        k[4] = bp * ux;
        k[5] = bp * uy;
        k[6] = m.cx[g];
        k[7] = m.cy[g];
    }
    return mp.seeds(coef, gX, gY);
}

int rtb_adjoint_destroy(rtb_adjoint* c) {
    if (!c) return RTB_OK;
    DeviceGuard dg(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->mem) cudaFree(c->mem);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return RTB_OK;
}

}  // extern "C"
