// engine.cu -- C ABI: engine state, scheme preparation and the drop-in calls
// of common-lib/rt_engine_func.h (host arrays in and out, synchronous).
//
// Each drop-in call copies the arrays it reads to the device, runs one
// kernel and copies back what the reference's call returns; the copies and
// the kernel are ordered on the library stream, the temporaries come from the
// stream-ordered pool (no cudaMalloc/cudaFree per call as in
// rt_cuda_engine_common.cu:72-155).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "engine.cuh"
#include "jit.h"

namespace rtb {

Engine& engine() {
    static Engine e;
    return e;
}

// The fault hook (rtb_fail_allocations): allocations to let through, then
// allocations to fail.
static std::atomic<int> g_alloc_skip{0}, g_alloc_fail{0};

static bool take_one(std::atomic<int>& c) {
    int n = c.load();
    while (n > 0)
        if (c.compare_exchange_weak(n, n - 1)) return true;
    return false;
}

bool injected_alloc_failure() {
    if (g_alloc_fail.load() <= 0) return false;
    if (take_one(g_alloc_skip)) return false;
    return take_one(g_alloc_fail);
}

cudaError_t dev_malloc(void** p, size_t bytes) {
    if (injected_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

int ensure_init() {
    Engine& e = engine();
    if (e.inited) return RTB_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return RTB_INIT_FAILED;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return RTB_INIT_FAILED;
    if (prop.major < 10) return RTB_INIT_FAILED;  // built for sm_100a only
    e.device = dev;
    e.sm_count = prop.multiProcessorCount;
    e.max_smem_optin = (int)prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking) != cudaSuccess) return RTB_INIT_FAILED;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~0ull;  // keep freed blocks for reuse instead of returning them to the driver
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    e.inited = true;
    return RTB_OK;
}

// ---------------------------------------------------------------------------
// Scheme preparation

double scheme_angle_rad(double deg) {
    double rad = deg * K_DEG2RAD;   // Surface::SetAngles (surface.cpp:201)
    double back = rad / K_DEG2RAD;  // Surface::GetAngles (surface.cpp:227)
    return back * K_DEG2RAD;        // Beam::Transform (beam.cpp:609-611)
}

// Translation and the rotations' host sin/cos (rt_cuda_engine_beam.cu:431-533).
void transform_constants(const double ang[3], const double dist[3], DevSurface& s) {
    for (int i = 0; i < 3; ++i) s.dist[i] = dist[i];
    s.translate = (dist[2] != 0.0) || (dist[0] != 0.0) || (dist[1] != 0.0);
    s.rot_mask = 0;
    for (int i = 0; i < 3; ++i) {
        if (ang[i] != 0) {
            s.rot_mask |= 1 << i;
            s.sinA[i] = std::sin(ang[i]);
            s.cosA[i] = std::cos(ang[i]);
        } else {
            s.sinA[i] = 0.0;
            s.cosA[i] = 1.0;
        }
    }
}

// copy_surf_params (rt_cuda_engine_surface.cu:108-148) and the dispatch of
// engine_intersection_cycle (surface.cu:593-636).
int surface_from_params(int cls, const double* params, DevSurface& s) {
    std::memset(&s, 0, sizeof(s));
    s.cls = cls;
    s.grating_index = -1;
    if (cls == RTB_AUX_CLASS) {
        s.kind = IS_NONE;
        s.k1 = 1.0;
        return RTB_OK;
    }
    if (cls != RTB_PLANE && cls != RTB_CONIC && cls != RTB_TORIC) return RTB_BAD_VALUE;
    if (!params) return RTB_BAD_VALUE;
    s.c = params[0];
    s.k1 = params[1] + 1;
    double nn = params[2];
    if (!(nn >= 0) || nn > RTB_MAX_POLY) return RTB_BAD_VALUE;
    s.n_poly = (int)(size_t)nn;
    for (int i = 0; i < s.n_poly; ++i) s.poly[i] = params[3 + i];
    s.cR = (cls == RTB_TORIC) ? params[3 + s.n_poly] : 0.0;
    if (cls == RTB_PLANE) {
        s.kind = IS_PLANE;
    } else if (cls == RTB_CONIC) {
        size_t NN = (size_t)params[2];
        if (NN == 0) {
            if (params[0] == 0) s.kind = IS_PLANE;
            else if (params[1] == -1) s.kind = IS_PARABOLOID;
            else s.kind = IS_CONIC;
        } else {
            s.kind = (params[0] == 0) ? IS_ITER_POLY : IS_ITER_CONIC;
        }
    } else {
        s.kind = IS_TORIC;
    }
    return RTB_OK;
}

bool KnotBuf::append(const double* v, size_t k) {
    if (vec) {
        vec->insert(vec->end(), v, v + k);
        return true;
    }
    if (n + k > cap) return false;
    for (size_t i = 0; i < k; ++i) fixed[n + i] = v[i];
    n += k;
    return true;
}

// Append a table to the knot buffer: [x(n) y(n) y2(n)], or [0, y0, 0] for a
// single value.  RTB_BAD_VALUE for a malformed table or a full fixed buffer.
int add_table(const rtb_table* t, KnotBuf& knots, int32_t& off, int32_t& cnt) {
    if (!t || t->n == 0 || !t->y) return RTB_BAD_VALUE;
    off = (int32_t)knots.size();
    if (t->n == 1) {
        cnt = 1;
        const double v[3] = {0.0, t->y[0], 0.0};
        return knots.append(v, 3) ? RTB_OK : RTB_BAD_VALUE;
    }
    if (t->n < 4 || t->n > RTB_MAX_KNOTS || !t->x || !t->y2) return RTB_BAD_VALUE;
    cnt = (int32_t)t->n;
    if (!knots.append(t->x, t->n) || !knots.append(t->y, t->n) || !knots.append(t->y2, t->n)) return RTB_BAD_VALUE;
    return RTB_OK;
}

int add_table(const rtb_table* t, std::vector<double>& knots, int32_t& off, int32_t& cnt) {
    KnotBuf kb(knots);
    return add_table(t, kb, off, cnt);
}

// The sag range of an even asphere over its circular pass aperture, for the
// mixed engine's test that a ray cannot meet the surface inside the aperture
// (mx::asphere_isect).  Points of the aperture (radius R about the centre c)
// lie at radii [max(0, |c| - R), |c| + R] from the axis; the sag
// c r^2 / (1 + sqrt(1 - k1 c^2 r^2)) + sum a_i r^(2i) is sampled there at 4097
// radii and the range widened by 1 % of its width plus 1 um, far more than
// the sag moves between samples.  No bounds where the base conic has no
// surface inside that radius.
void asphere_sag_bounds(DevSurface& s) {
    s.sag_cull = 0;
    s.sag_lo = s.sag_hi = 0.0;
    if (s.kind != IS_ITER_CONIC && s.kind != IS_ITER_POLY) return;
    if (s.shape != RTB_CIRCLE || s.type == RTB_SHADE || !(s.size[0] > 0)) return;
    const double rc = std::hypot(s.center[0], s.center[1]);
    const double r_lo = std::max(0.0, rc - s.size[0]), r_hi = rc + s.size[0];
    double lo = 1e300, hi = -1e300;
    const int n = 4097;
    for (int i = 0; i < n; ++i) {
        const double r = r_lo + (r_hi - r_lo) * i / (n - 1);
        const double r2 = r * r;
        double z = 0.0;
        if (s.kind == IS_ITER_CONIC) {
            const double q = 1.0 - s.k1 * s.c * s.c * r2;
            if (!(q >= 0.0)) return;
            z = s.c * r2 / (1.0 + std::sqrt(q));
        }
        double p = 0.0;
        for (int k = s.n_poly; k >= 1; --k) p = (p + s.poly[k - 1]) * r2;
        z += p;
        if (!std::isfinite(z)) return;
        lo = std::min(lo, z);
        hi = std::max(hi, z);
    }
    const double m = 0.01 * (hi - lo) + 1e-3;
    s.sag_lo = lo - m;
    s.sag_hi = hi + m;
    s.sag_cull = 1;
}

void mixed_constants(DevSurface& s) {
    asphere_sag_bounds(s);
    s.inv_c = (s.c != 0.0) ? 1.0 / s.c : 0.0;
    s.inv_gr = (s.gr_const != 0.0) ? 1.0 / s.gr_const : 0.0;
    s.f_c = (float)s.c;
    s.f_k1 = (float)s.k1;
    s.f_cR = (float)s.cR;
    s.f_inv_c = (float)s.inv_c;
    s.f_sag_lo = (float)s.sag_lo;
    s.f_sag_hi = (float)s.sag_hi;
    s.f_size0 = (float)s.size[0];
    s.f_pad = 0.0f;
    for (int i = 0; i < RTB_MAX_POLY; ++i) {
        s.f_poly[i] = (float)s.poly[i];
        s.f_ipoly[i] = (float)(i + 1) * (float)s.poly[i];
    }
}

// Every number a surface contributes to a trace is finite: a NaN or an
// infinity in the scheme is a bad request, refused before any launch (the
// reference would trace it into NaN rays).
static bool surface_finite(const rtb_surface& in) {
    const double nn = in.params[2];
    if (!std::isfinite(in.params[0]) || !std::isfinite(in.params[1]) || !std::isfinite(nn)) return false;
    const int used = 3 + ((nn >= 0 && nn <= RTB_MAX_POLY) ? (int)nn : 0) + (in.cls == RTB_TORIC ? 1 : 0);
    for (int i = 3; i < used && i < RTB_MAX_PARAMS; ++i)
        if (!std::isfinite(in.params[i])) return false;
    for (int i = 0; i < 3; ++i)
        if (!std::isfinite(in.distance[i]) || !std::isfinite(in.angles_deg[i])) return false;
    for (int i = 0; i < 2; ++i)
        if (!std::isfinite(in.size[i]) || !std::isfinite(in.center[i])) return false;
    return in.type != RTB_GRATING || std::isfinite(in.gr_const);
}

int prepare_surface(const rtb_surface& in, DevSurface& s, KnotBuf& knots) {
    if (in.type != RTB_AUX_TYPE && !surface_finite(in)) return RTB_BAD_VALUE;
    bool non_aux = in.type != RTB_AUX_TYPE;
    int st = surface_from_params(non_aux ? in.cls : RTB_AUX_CLASS, in.params, s);
    if (st != RTB_OK) return st;
    s.cls = in.cls;
    s.type = in.type;
    s.shape = in.shape;
    s.gr_type = in.grating_type;
    s.non_aux = non_aux;
    if (!non_aux) s.kind = IS_NONE;
    s.order = in.order;
    s.gr_const = in.gr_const;
    if (in.type < RTB_MIRROR || in.type > RTB_AUX_TYPE) return RTB_BAD_VALUE;
    if (in.shape != RTB_CIRCLE && in.shape != RTB_RECTANGLE) return RTB_BAD_VALUE;
    if (in.type == RTB_GRATING && in.grating_type != RTB_REFLECTIVE && in.grating_type != RTB_TRANSPARENT)
        return RTB_BAD_VALUE;
    double ang[3];
    for (int i = 0; i < 3; ++i) ang[i] = scheme_angle_rad(in.angles_deg[i]);
    transform_constants(ang, in.distance, s);
    for (int i = 0; i < 2; ++i) {
        s.size[i] = in.size[i];
        s.center[i] = in.center[i];
    }
    mixed_constants(s);
    s.n1_off = s.n2_off = 0;
    s.n1_n = s.n2_n = 1;
    if (in.type == RTB_LENS || in.type == RTB_GRATING) {
        st = add_table(&in.n2, knots, s.n2_off, s.n2_n);
        if (st != RTB_OK) return st;
        if (in.type == RTB_LENS || in.grating_type == RTB_TRANSPARENT) {
            st = add_table(&in.n1, knots, s.n1_off, s.n1_n);
            if (st != RTB_OK) return st;
        }
    }
    return RTB_OK;
}

// The rotations of one surface's transform applied to v, in the kernels'
// order: about y (X,Z), about x (Y,Z), about z (X,Y) (beam.cu:437-518).
static void rotate_by(const DevSurface& s, double v[3]) {
    if (s.rot_mask & 1) {
        const double e = v[0] * s.cosA[0] - v[2] * s.sinA[0];
        v[2] = v[0] * s.sinA[0] + v[2] * s.cosA[0];
        v[0] = e;
    }
    if (s.rot_mask & 2) {
        const double e = v[1] * s.cosA[1] - v[2] * s.sinA[1];
        v[2] = v[1] * s.sinA[1] + v[2] * s.cosA[1];
        v[1] = e;
    }
    if (s.rot_mask & 4) {
        const double e = v[0] * s.cosA[2] - v[1] * s.sinA[2];
        v[1] = v[0] * s.sinA[2] + v[1] * s.cosA[2];
        v[0] = e;
    }
}

// The FP32-state engine's transforms: from the frame of one non-Aux surface
// to the next (P' = M P + off, D' = M D), each surface's translation and
// rotations and those of the Aux surfaces in between composed in FP64 here.
static void fp32_transforms(DevScheme& sch) {
    double M[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, off[3] = {0, 0, 0};
    bool first = true;
    for (int k = 0; k < sch.n_surfaces; ++k) {
        DevSurface& s = sch.s[k];
        // P -> R_k (M P + off - d_k): the columns of M and the offset rotate
        for (int c = 0; c < 3; ++c) {
            double v[3] = {M[c], M[3 + c], M[6 + c]};
            rotate_by(s, v);
            M[c] = v[0];
            M[3 + c] = v[1];
            M[6 + c] = v[2];
        }
        double o[3] = {off[0] - s.dist[0], off[1] - s.dist[1], off[2] - s.dist[2]};
        rotate_by(s, o);
        for (int i = 0; i < 3; ++i) off[i] = o[i];
        if (!s.non_aux) continue;
        bool ident = true;
        for (int i = 0; i < 9; ++i) {
            s.m32[i] = make_float2((float)M[i], (float)M[i]);
            ident = ident && M[i] == ((i % 4 == 0) ? 1.0 : 0.0);
        }
        s.rot32 = ident ? 0 : 1;
        s.first32 = first ? 1 : 0;
        for (int i = 0; i < 3; ++i) s.off32[i] = off[i];
        if (first) {
            for (int i = 0; i < 9; ++i) sch.m0[i] = M[i];
            for (int i = 0; i < 3; ++i) sch.off0[i] = off[i];
            first = false;
        }
        for (int i = 0; i < 9; ++i) M[i] = (i % 4 == 0) ? 1.0 : 0.0;
        off[0] = off[1] = off[2] = 0.0;
    }
    bool tail = false;
    for (int i = 0; i < 9; ++i) {
        sch.tail_m[i] = M[i];
        tail = tail || M[i] != ((i % 4 == 0) ? 1.0 : 0.0);
    }
    for (int i = 0; i < 3; ++i) {
        sch.tail_off[i] = off[i];
        tail = tail || off[i] != 0.0;
    }
    sch.tail_on = tail ? 1 : 0;
}

void beam_frame(const DevScheme& sch, const double center[3], DevBeam& d) {
    for (int i = 0; i < 3; ++i) {
        d.origin[i] = center[i];
        d.off0[i] = sch.m0[3 * i] * center[0] + sch.m0[3 * i + 1] * center[1] + sch.m0[3 * i + 2] * center[2] +
                    sch.off0[i];
    }
}

int prepare_scheme_into(const rtb_surface* surf, size_t n, uint32_t fixes, int renorm_lost, DevScheme& sch,
                        KnotBuf& knots) {
    if (!surf || n == 0 || n > RTB_MAX_SURFACES) return RTB_BAD_VALUE;
    std::memset(&sch, 0, sizeof(sch));
    const double unit[3] = {0.0, 1.0, 0.0};  // offset 0: a harmless single value for unused tables
    if (!knots.append(unit, 3)) return RTB_BAD_VALUE;
    int ng = 0, nonaux = 0;
    for (size_t k = 0; k < n; ++k) {
        DevSurface& s = sch.s[k];
        int st = prepare_surface(surf[k], s, knots);
        if (st != RTB_OK) return st;
        s.grating_index = (s.type == RTB_GRATING) ? ng++ : -1;
        if (s.non_aux) ++nonaux;
        s.surfaces_upto = nonaux;
    }
    if (ng > RTB_MAX_GRATINGS) return RTB_BAD_VALUE;
    for (size_t k = 0; k < n; ++k) {
        int cnt = sch.s[k].non_aux ? 1 : 0;
        for (size_t j = k + 1; j < n; ++j) cnt += 1 + (sch.s[j].non_aux ? 1 : 0);
        sch.s[k].renorm_after = cnt;
    }
    const double* kn = knots.data();
    // identical tables share one copy (a lens's glass is the index after its
    // front surface and before its back surface), and a table on a uniform
    // grid records its inverse spacing for the mixed engine's direct lookup
    auto same = [&](int32_t o1, int32_t o2, int32_t cnt) {
        const int32_t len = (cnt == 1) ? 3 : 3 * cnt;
        for (int32_t i = 0; i < len; ++i)
            if (kn[o1 + i] != kn[o2 + i]) return false;
        return true;
    };
    auto inv_spacing = [&](int32_t off, int32_t cnt) {
        if (cnt < 2) return 0.0;
        const double* x = kn + off;
        const double h = (x[cnt - 1] - x[0]) / (cnt - 1);
        if (!(h > 0)) return 0.0;
        for (int32_t i = 0; i < cnt; ++i)
            if (std::fabs(x[i] - (x[0] + i * h)) > 1e-9 * h) return 0.0;
        return 1.0 / h;
    };
    for (size_t k = 0; k < n; ++k) {
        DevSurface& s = sch.s[k];
        int32_t* offs[2] = {&s.n1_off, &s.n2_off};
        int32_t cnts[2] = {s.n1_n, s.n2_n};
        for (int t = 0; t < 2; ++t) {
            for (size_t j = 0; j <= k; ++j) {
                const DevSurface& e = sch.s[j];
                const int32_t eo[2] = {e.n1_off, e.n2_off}, ec[2] = {e.n1_n, e.n2_n};
                bool done = false;
                for (int u = 0; u < 2 && !done; ++u) {
                    if (j == k && u >= t) break;
                    if (ec[u] == cnts[t] && eo[u] != *offs[t] && same(eo[u], *offs[t], cnts[t])) {
                        *offs[t] = eo[u];
                        done = true;
                    }
                }
                if (done) break;
            }
        }
        s.n1_invh = inv_spacing(s.n1_off, s.n1_n);
        s.n2_invh = inv_spacing(s.n2_off, s.n2_n);
    }
    sch.n_surfaces = (int32_t)n;
    sch.n_knots = (int32_t)knots.size();
    sch.fixes = fixes;
    sch.renorm_lost = renorm_lost;
    fp32_transforms(sch);
    return RTB_OK;
}

int prepare_scheme(const rtb_surface* surf, size_t n, uint32_t fixes, int renorm_lost, PreparedScheme& out) {
    out.knots.clear();
    KnotBuf kb(out.knots);
    return prepare_scheme_into(surf, n, fixes, renorm_lost, out.sch, kb);
}

// Natural cubic spline second derivatives: the sequential algorithm of
// Numerical Recipes that rt_cuda_engine_spline.cu:43-145 intends (its
// kernel runs the recurrence in parallel and races); 4..1024 knots run in
// well under a microsecond on the host.
static void spline_second_derivatives(size_t N, const double* x, const double* y, double* y2) {
    std::vector<double> u(N, 0.0);
    y2[0] = 0.0;
    y2[N - 1] = 0.0;
    for (size_t i = 1; i + 1 < N; ++i) {
        double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
        double p = sig * y2[i - 1] + 2.0;
        y2[i] = (sig - 1.0) / p;
        u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
        u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
    }
    for (size_t k = N - 2; k > 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
}

// ---------------------------------------------------------------------------
// Drop-in helpers

namespace {

// Device copies of up to 8 double arrays and one flag array, from one pool
// allocation.
struct Staged {
    DevBuf buf;
    double* d[8] = {nullptr};
    char* flag = nullptr;
    unsigned long long* counter = nullptr;
    unsigned* err = nullptr;
    int init(size_t n, int n_double, bool with_flag, cudaStream_t st) {
        size_t bytes = 64 + n_double * n * sizeof(double) + (with_flag ? n + 16 : 0);
        int s = buf.alloc(bytes, st);
        if (s != RTB_OK) return s;
        char* p = buf.as<char>();
        counter = reinterpret_cast<unsigned long long*>(p);
        err = reinterpret_cast<unsigned*>(p + 8);
        p += 64;
        for (int i = 0; i < n_double; ++i) {
            d[i] = reinterpret_cast<double*>(p);
            p += n * sizeof(double);
        }
        if (with_flag) flag = p;
        RTB_CUDA_TRY(cudaMemsetAsync(buf.p, 0, 64, st));
        return RTB_OK;
    }
};

int h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return RTB_OK;
    RTB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return RTB_OK;
}

int d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return RTB_OK;
    RTB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    return RTB_OK;
}

int finish(cudaStream_t st, const unsigned* d_err, size_t* n_bad, const unsigned long long* d_counter) {
    unsigned long long cnt = 0;
    unsigned err = 0;
    if (d_counter) RTB_CUDA_TRY(cudaMemcpyAsync(&cnt, d_counter, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    if (d_err) RTB_CUDA_TRY(cudaMemcpyAsync(&err, d_err, sizeof(err), cudaMemcpyDeviceToHost, st));
    RTB_CUDA_TRY(cudaStreamSynchronize(st));
    RTB_CUDA_TRY(cudaGetLastError());
    if (err & DEV_ERR_OUT_OF_RANGE) return RTB_OUT_OF_RANGE;
    if (err) return RTB_BAD_VALUE;
    if (n_bad) *n_bad += (size_t)cnt;
    return RTB_OK;
}

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" RTB_API int rtb_fail_allocations(uint32_t after, uint32_t count) {
    rtb::g_alloc_fail.store(0);
    rtb::g_alloc_skip.store((int)(after > 1000000u ? 1000000u : after));
    rtb::g_alloc_fail.store((int)(count > 1000000u ? 1000000u : count));
    return RTB_OK;
}

extern "C" {

int rtb_init(void) {
    Lock l;
    return ensure_init();
}

int rtb_info(char* buf, size_t buflen) {
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, engine().device) != cudaSuccess) return RTB_FAILED;
    std::string s = "B200 ray-tracing engine (sm_100a)\n";
    s += std::string("Device name: ") + prop.name + "\n";
    s += "Computing ability: " + std::to_string(prop.major) + "." + std::to_string(prop.minor) + "\n";
    s += "Global memory: " + std::to_string(prop.totalGlobalMem) + "\n";
    s += "Number of multiprocessors: " + std::to_string(prop.multiProcessorCount) + "\n";
    s += "NVRTC (scheme-specialised kernels): " + nvrtc_info() + "\n";
    if (!buf || buflen == 0) return RTB_BAD_VALUE;
    std::snprintf(buf, buflen, "%s", s.c_str());
    return RTB_OK;
}

int rtb_spline_init(size_t n, const double* x, const double* y, double* y2) {
    if (n < 4 || !x || !y || !y2) return RTB_BAD_VALUE;
    spline_second_derivatives(n, x, y, y2);
    return RTB_OK;
}

double* rtb_alocate_vector(size_t n_elem) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, sizeof(double) * (n_elem ? n_elem : 1), cudaHostAllocPortable) != cudaSuccess) return nullptr;
    return static_cast<double*>(p);
}

void rtb_free_vector(double* data) {
    if (data) cudaFreeHost(data);
}

int rtb_beam_random(int shape, const double* params, const double* center, size_t n, double* X, double* Y, double* Z,
                    uint64_t seed, uint64_t first_ray) {
    if (shape != RTB_CIRCLE || !params || !center) return RTB_BAD_VALUE;
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 3, false, s)) != RTB_OK) return st;
    k_beam_random<<<grid_for(n, 256, 8), 256, 0, s>>>(n, params[1], params[2], center[0], center[1], center[2], seed,
                                                        first_ray, g.d[0], g.d[1], g.d[2]);
    double* out[3] = {X, Y, Z};
    for (int i = 0; i < 3; ++i)
        if ((st = d2h(out[i], g.d[i], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

// conic_cosins_kernel (rt_cuda_engine_beam.cu:586-611): cZ = cos(a/2),
// (cX, cY) = sin(a/2) (cos, sin)(atan2(Y, X)).  Evaluated on the host: it is
// not on the benchmark path and uses transcendental functions per ray.
int rtb_beam_conic_cosins(size_t n, double conic_angle, const double* X, const double* Y, double* cX, double* cY,
                          double* cZ) {
    if (n && (!X || !Y || !cX || !cY || !cZ)) return RTB_BAD_VALUE;
    double cc = std::cos(conic_angle / 2.0), sc = std::sin(conic_angle / 2.0);
    for (size_t i = 0; i < n; ++i) {
        double phi = std::atan2(Y[i], X[i]);
        cZ[i] = cc;
        cX[i] = sc * std::cos(phi);
        cY[i] = sc * std::sin(phi);
    }
    return RTB_OK;
}

// gauss_cosins_kernel (rt_cuda_engine_beam.cu:952-991) re-derived: two
// rotations by normal deviates of standard deviation tan(sigma), sigma the
// FWHM in arcsec converted to radians (beam.cu:1099).  Host-side, seeded.
int rtb_beam_gauss_cosins(size_t n, double fwhm, double* cX, double* cY, double* cZ, uint64_t seed) {
    if (n && (!cX || !cY || !cZ)) return RTB_BAD_VALUE;
    double stddev = fwhm / 2.35482 * K_RT_PI / 180 / 3600;
    double tg = std::tan(stddev);
    uint64_t state = seed * 0x9E3779B97F4A7C15ull + 1;
    auto next_u = [&]() {
        state ^= state >> 12;
        state ^= state << 25;
        state ^= state >> 27;
        return ((state * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0) + 1e-300;
    };
    for (size_t i = 0; i < n; ++i) {
        double u1 = next_u(), u2 = next_u();
        double rad = std::sqrt(-2.0 * std::log(u1));
        double gx = tg * rad * std::cos(6.283185307179586 * u2);
        double gy = tg * rad * std::sin(6.283185307179586 * u2);
        double x = 0.0, y = 0.0, z = 1.0;
        double cs = 1.0 / std::sqrt(1.0 + gx * gx);
        double sn = (std::signbit(gx) ? -1.0 : 1.0) * (gx == 0 ? 0.0 : 1.0 / std::sqrt(1.0 + 1.0 / gx / gx));
        y = -sn * z;
        z = cs * z;
        cs = 1.0 / std::sqrt(1.0 + gy * gy);
        sn = (std::signbit(gy) ? -1.0 : 1.0) * (gy == 0 ? 0.0 : 1.0 / std::sqrt(1.0 + 1.0 / gy / gy));
        x = -sn * z;
        z = cs * z;
        cX[i] = x;
        cY[i] = y;
        cZ[i] = z;
    }
    return RTB_OK;
}

int rtb_uniform_range_beam(size_t n, const double* range, double* lambda) {
    if (!range || (n && !lambda)) return RTB_BAD_VALUE;
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    double d_l = (range[1] - range[0]) / (n - 1);  // rt_cuda_engine_beam.cu:726
    Staged g;
    if ((st = g.init(n, 1, false, s)) != RTB_OK) return st;
    k_uniform_range<<<grid_for(n, 256, 8), 256, 0, s>>>(n, range[0], d_l, g.d[0]);
    if ((st = d2h(lambda, g.d[0], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

int rtb_random_range_beam(size_t n, const double* range, double* lambda, uint64_t seed) {
    if (!range || (n && !lambda)) return RTB_BAD_VALUE;
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 1, false, s)) != RTB_OK) return st;
    k_random_range<<<grid_for(n, 256, 8), 256, 0, s>>>(n, range[0], range[1], seed, g.d[0]);
    if ((st = d2h(lambda, g.d[0], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

int rtb_beam_transform(size_t n, const double* angles, const double* dist, double* X, double* Y, double* Z,
                       double* cX, double* cY, double* cZ) {
    if (!angles || !dist) return RTB_BAD_VALUE;
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    DevSurface ds;
    std::memset(&ds, 0, sizeof(ds));
    transform_constants(angles, dist, ds);
    Staged g;
    if ((st = g.init(n, 6, false, s)) != RTB_OK) return st;
    double* a[6] = {X, Y, Z, cX, cY, cZ};
    for (int i = 0; i < 6; ++i)
        if ((st = h2d(g.d[i], a[i], n * sizeof(double), s)) != RTB_OK) return st;
    k_transform<<<grid_for(n, 256, 8), 256, 0, s>>>(n, ds, g.d[0], g.d[1], g.d[2], g.d[3], g.d[4], g.d[5]);
    for (int i = 0; i < 6; ++i)
        if ((st = d2h(a[i], g.d[i], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

static int intersection_impl(int cls, const double* params, size_t n, double* X, double* Y, double* Z, double* cX,
                             double* cY, double* cZ, size_t* n_bad, char* flag, uint32_t fixes) {
    if (!n_bad) return RTB_BAD_VALUE;
    if (cls == RTB_AUX_CLASS || n == 0) return RTB_OK;  // surface.cu:634-635
    DevSurface ds;
    int st = surface_from_params(cls, params, ds);
    if (st != RTB_OK) return st;
    Lock l;
    if ((st = ensure_init()) != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 6, true, s)) != RTB_OK) return st;
    double* a[6] = {X, Y, Z, cX, cY, cZ};
    for (int i = 0; i < 6; ++i)
        if ((st = h2d(g.d[i], a[i], n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.flag, flag, n, s)) != RTB_OK) return st;
    k_intersect<<<grid_for(n, 256, 8), 256, 0, s>>>(n, ds, fixes, g.d[0], g.d[1], g.d[2], g.d[3], g.d[4], g.d[5],
                                                      g.flag, g.counter);
    for (int i = 0; i < 3; ++i)
        if ((st = d2h(a[i], g.d[i], n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = d2h(flag, g.flag, n, s)) != RTB_OK) return st;
    return finish(s, g.err, n_bad, g.counter);
}

int rtb_surface_intersection(int cls, const double* params, size_t n, double* X, double* Y, double* Z, double* cX,
                             double* cY, double* cZ, size_t* n_bad, char* flag) {
    return intersection_impl(cls, params, n, X, Y, Z, cX, cY, cZ, n_bad, flag, 0);
}

int rtb_surface_intersection_fix(int cls, const double* params, size_t n, double* X, double* Y, double* Z,
                                 double* cX, double* cY, double* cZ, size_t* n_bad, char* flag, uint32_t fixes) {
    return intersection_impl(cls, params, n, X, Y, Z, cX, cY, cZ, n_bad, flag, fixes);
}

int rtb_surface_reflection(int cls, const double* params, size_t n, double* X, double* Y, double* Z, double* cX,
                           double* cY, double* cZ) {
    if (n == 0) return RTB_OK;
    DevSurface ds;
    int st = surface_from_params(cls, params, ds);
    if (st != RTB_OK) return st;
    Lock l;
    if ((st = ensure_init()) != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 6, false, s)) != RTB_OK) return st;
    double* a[6] = {X, Y, Z, cX, cY, cZ};
    for (int i = 0; i < 6; ++i)
        if ((st = h2d(g.d[i], a[i], n * sizeof(double), s)) != RTB_OK) return st;
    k_reflect<<<grid_for(n, 256, 8), 256, 0, s>>>(n, ds, g.d[0], g.d[1], g.d[2], g.d[3], g.d[4], g.d[5]);
    for (int i = 3; i < 6; ++i)
        if ((st = d2h(a[i], g.d[i], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

// Refraction (type Lens) or diffraction (type Grating) over host arrays.
static int action_impl(int type, int cls, int gr_type, const double* params, long order, double gr_const, size_t n,
                       double* X, double* Y, double* Z, double* cX, double* cY, double* cZ, const double* lambda,
                       const rtb_table* n1, const rtb_table* n2, size_t* n_bad, char* flag) {
    if (!n_bad) return RTB_BAD_VALUE;
    if (n == 0) return RTB_OK;
    DevSurface ds;
    int st = surface_from_params(cls, params, ds);
    if (st != RTB_OK) return st;
    ds.type = type;
    ds.gr_type = gr_type;
    ds.gr_const = gr_const;
    std::vector<double> knots = {0.0, 1.0, 0.0};
    if ((st = add_table(n2, knots, ds.n2_off, ds.n2_n)) != RTB_OK) return st;
    if (type == RTB_LENS || gr_type == RTB_TRANSPARENT) {
        if ((st = add_table(n1, knots, ds.n1_off, ds.n1_n)) != RTB_OK) return st;
    }
    Lock l;
    if ((st = ensure_init()) != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 7, true, s)) != RTB_OK) return st;
    DevBuf kb;
    if ((st = kb.alloc(knots.size() * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(kb.p, knots.data(), knots.size() * sizeof(double), s)) != RTB_OK) return st;
    double* a[6] = {X, Y, Z, cX, cY, cZ};
    for (int i = 0; i < 6; ++i)
        if ((st = h2d(g.d[i], a[i], n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.d[6], lambda, n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.flag, flag, n, s)) != RTB_OK) return st;
    k_action<<<grid_for(n, 256, 8), 256, 0, s>>>(n, ds, kb.as<double>(), (long long)order, g.d[6], g.d[0], g.d[1],
                                                   g.d[2], g.d[3], g.d[4], g.d[5], g.flag, g.counter, g.err);
    for (int i = 3; i < 6; ++i)
        if ((st = d2h(a[i], g.d[i], n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = d2h(flag, g.flag, n, s)) != RTB_OK) return st;
    return finish(s, g.err, n_bad, g.counter);
}

int rtb_surface_refraction(int cls, const double* params, size_t n, double* X, double* Y, double* Z, double* cX,
                           double* cY, double* cZ, const double* lambda, const rtb_table* n1, const rtb_table* n2,
                           size_t* n_bad, char* flag) {
    return action_impl(RTB_LENS, cls, RTB_REFLECTIVE, params, 0, 0.0, n, X, Y, Z, cX, cY, cZ, lambda, n1, n2, n_bad,
                       flag);
}

int rtb_surface_diffration(int cls, int gr_type, const double* params, long diff_order, double gr_constant, size_t n,
                           double* X, double* Y, double* Z, double* cX, double* cY, double* cZ, const double* lambda,
                           const rtb_table* n1, const rtb_table* n2, size_t* n_bad, char* flag) {
    if (gr_type != RTB_REFLECTIVE && gr_type != RTB_TRANSPARENT) return RTB_BAD_VALUE;  // surface.cu:1637,1706
    return action_impl(RTB_GRATING, cls, gr_type, params, diff_order, gr_constant, n, X, Y, Z, cX, cY, cZ, lambda, n1,
                       n2, n_bad, flag);
}

int rtb_surface_QE(size_t n, const double* lambda, double* spec, const rtb_table* qe) {
    if (n == 0) return RTB_OK;
    std::vector<double> knots;
    int32_t off, cnt;
    int st = add_table(qe, knots, off, cnt);
    if (st != RTB_OK) return st;
    Lock l;
    if ((st = ensure_init()) != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 2, false, s)) != RTB_OK) return st;
    DevBuf kb;
    if ((st = kb.alloc(knots.size() * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(kb.p, knots.data(), knots.size() * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.d[0], lambda, n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.d[1], spec, n * sizeof(double), s)) != RTB_OK) return st;
    k_surface_qe<<<grid_for(n, 256, 8), 256, 0, s>>>(n, g.d[0], g.d[1], kb.as<double>(), off, cnt, g.err);
    if ((st = d2h(spec, g.d[1], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, g.err, nullptr, nullptr);
}

int rtb_normalize(size_t n, double* cX, double* cY, double* cZ) {
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 3, false, s)) != RTB_OK) return st;
    double* a[3] = {cX, cY, cZ};
    for (int i = 0; i < 3; ++i)
        if ((st = h2d(g.d[i], a[i], n * sizeof(double), s)) != RTB_OK) return st;
    k_normalize<<<grid_for(n, 256, 8), 256, 0, s>>>(n, g.d[0], g.d[1], g.d[2]);
    for (int i = 0; i < 3; ++i)
        if ((st = d2h(a[i], g.d[i], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

int rtb_apply_constrains(int shade, int shape, const double* size, const double* center, size_t n, const double* X,
                         const double* Y, char* flag, size_t* n_bad) {
    if (!size || !center || !n_bad) return RTB_BAD_VALUE;
    if (shape != RTB_CIRCLE && shape != RTB_RECTANGLE) return RTB_BAD_VALUE;
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 2, true, s)) != RTB_OK) return st;
    if ((st = h2d(g.d[0], X, n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.d[1], Y, n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.flag, flag, n, s)) != RTB_OK) return st;
    k_aperture<<<grid_for(n, 256, 8), 256, 0, s>>>(n, shade, shape, size[0], shape == RTB_RECTANGLE ? size[1] : 0.0,
                                                     center[0], center[1], g.d[0], g.d[1], g.flag, g.counter);
    if ((st = d2h(flag, g.flag, n, s)) != RTB_OK) return st;
    return finish(s, nullptr, n_bad, g.counter);
}

int rtb_ccd_coordinates(size_t n, const double* X, const double* Y, double xsize, double ysize, double xpix,
                        double ypix, unsigned int* ccd_X, unsigned int* ccd_Y) {
    if (n == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 3, false, s)) != RTB_OK) return st;
    if ((st = h2d(g.d[0], X, n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.d[1], Y, n * sizeof(double), s)) != RTB_OK) return st;
    unsigned* ix = reinterpret_cast<unsigned*>(g.d[2]);
    unsigned* iy = ix + n;
    k_ccd_coords<<<grid_for(n, 256, 8), 256, 0, s>>>(n, g.d[0], g.d[1], xsize, ysize, xpix, ypix, ix, iy);
    if ((st = d2h(ccd_X, ix, n * sizeof(unsigned), s)) != RTB_OK) return st;
    if ((st = d2h(ccd_Y, iy, n * sizeof(unsigned), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

int rtb_compute_ccd_image(size_t n, const unsigned int* ccd_X, const unsigned int* ccd_Y, const double* lambda,
                          const rtb_table* qe, const rtb_table* spec, size_t xdim, size_t ydim, double xpix,
                          double ypix, double* image, uint64_t* n_outside) {
    if (!image || xdim == 0 || ydim == 0) return RTB_BAD_VALUE;
    if (xdim * ydim > 0xFFFFFFFFull) return RTB_BAD_VALUE;  // 32-bit pixel index (ccd.cu:224)
    std::vector<double> knots;
    int32_t qo, qn, so, sn;
    int st = add_table(qe, knots, qo, qn);
    if (st != RTB_OK) return st;
    if ((st = add_table(spec, knots, so, sn)) != RTB_OK) return st;
    Lock l;
    if ((st = ensure_init()) != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    size_t npix = xdim * ydim;
    DevBuf img, kb;
    if ((st = img.alloc(npix * sizeof(double), s)) != RTB_OK) return st;
    if ((st = kb.alloc(knots.size() * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(kb.p, knots.data(), knots.size() * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(img.p, image, npix * sizeof(double), s)) != RTB_OK) return st;
    Staged g;
    if ((st = g.init(n ? n : 1, 2, false, s)) != RTB_OK) return st;
    if (n) {
        unsigned* ix = reinterpret_cast<unsigned*>(g.d[1]);
        unsigned* iy = ix + n;
        if ((st = h2d(g.d[0], lambda, n * sizeof(double), s)) != RTB_OK) return st;
        if ((st = h2d(ix, ccd_X, n * sizeof(unsigned), s)) != RTB_OK) return st;
        if ((st = h2d(iy, ccd_Y, n * sizeof(unsigned), s)) != RTB_OK) return st;
        double pix_area = xpix * ypix * 1.0E-2;  // ccd.cu:360
        k_ccd_image<<<grid_for(n, 256, 8), 256, 0, s>>>(n, ix, iy, g.d[0], kb.as<double>(), qo, qn, so, sn, xdim, ydim,
                                                          pix_area, img.as<double>(), g.counter, g.err);
    }
    if ((st = d2h(image, img.p, npix * sizeof(double), s)) != RTB_OK) return st;
    size_t outside = 0;
    st = finish(s, g.err, &outside, g.counter);
    if (st == RTB_OK && n_outside) *n_outside += outside;
    return st;
}

}  // extern "C"

namespace rtb {
__global__ void k_grating_energy(size_t n, const double* lambda, long long order, double blaze, double alpha,
                                 double gamma, double gr_const, double rule_start, double rule_stop, double* energy);
}

extern "C" int rtb_grating_energy_distr(size_t n, const double* lambda, long order, double blaze_angle, double alpha,
                                        double gamma, double gr_const, double rule_start, double rule_stop,
                                        double* energy_distr) {
    if (n == 0) return RTB_OK;
    if (!lambda || !energy_distr) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    Staged g;
    if ((st = g.init(n, 2, false, s)) != RTB_OK) return st;
    if ((st = h2d(g.d[0], lambda, n * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(g.d[1], energy_distr, n * sizeof(double), s)) != RTB_OK) return st;
    k_grating_energy<<<grid_for(n, 256, 8), 256, 0, s>>>(n, g.d[0], (long long)order, blaze_angle, alpha, gamma,
                                                          gr_const, rule_start, rule_stop, g.d[1]);
    if ((st = d2h(energy_distr, g.d[1], n * sizeof(double), s)) != RTB_OK) return st;
    return finish(s, nullptr, nullptr, nullptr);
}

extern "C" int rtb_qe_curves(const rtb_qe_surface* surfaces, size_t n_surfaces, const double* rows, size_t n_rows,
                             size_t row_len, size_t n_lambda, double* lambda, double* qe) {
    if (n_rows == 0) return RTB_OK;
    if (!rows || !lambda || !qe || (n_surfaces && !surfaces) || n_lambda < 2 || row_len < 2) return RTB_BAD_VALUE;
    if (n_surfaces > (size_t)RTB_MAX_SURFACES || n_lambda > ((size_t)1 << 40) / n_rows) return RTB_BAD_VALUE;
    std::vector<QeSurface> qs(n_surfaces);
    std::vector<double> knots;
    size_t n_gratings = 0;
    for (size_t k = 0; k < n_surfaces; ++k) {
        const rtb_qe_surface& in = surfaces[k];
        QeSurface& o = qs[k];
        std::memset(&o, 0, sizeof(o));
        int st = add_table(&in.qe, knots, o.off, o.cnt);
        if (st != RTB_OK) return st;
        if (in.type == RTB_GRATING) {
            // Grating::SetRuleParams (surface.cpp:595-611): `x*deg2rad` expands
            // to x*RT_PI/180.0, evaluated left to right
            o.grating = 1;
            o.order = in.order;
            o.gr_const = in.gr_const;
            o.blaze = in.blaze_deg * K_RT_PI / 180.0;
            o.alpha = in.alpha_deg * K_RT_PI / 180.0;
            o.gamma = in.gamma_deg * K_RT_PI / 180.0;
            double a = in.rule_start, b = in.rule_stop;
            if (a < 0.0) a = 0.0;
            if (a > 1.0) a = 1.0;
            if (b < 0.0) b = 0.0;
            if (b > 1.0) b = 1.0;
            if (a >= b) return RTB_BAD_VALUE;
            o.rule_size = b - a;
            ++n_gratings;
        } else if (in.type != RTB_MIRROR && in.type != RTB_LENS && in.type != RTB_DETECTOR) {
            return RTB_BAD_VALUE;
        }
    }
    const int from_rows = n_rows > 1;
    if (from_rows && row_len < 2 + n_gratings) return RTB_BAD_VALUE;
    const size_t total = n_rows * n_lambda;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_rows = up(n_rows * row_len * sizeof(double)), b_s = up(qs.size() * sizeof(QeSurface) + 16),
                 b_k = up(knots.size() * sizeof(double) + 16), b_out = total * sizeof(double);
    DevBuf buf;
    if ((st = buf.alloc(256 + b_rows + b_s + b_k + 2 * up(b_out), s)) != RTB_OK) return st;
    char* p = buf.as<char>();
    unsigned* err = reinterpret_cast<unsigned*>(p);
    double* d_rows = reinterpret_cast<double*>(p + 256);
    QeSurface* d_s = reinterpret_cast<QeSurface*>(p + 256 + b_rows);
    double* d_k = reinterpret_cast<double*>(p + 256 + b_rows + b_s);
    double* d_l = reinterpret_cast<double*>(p + 256 + b_rows + b_s + b_k);
    double* d_q = reinterpret_cast<double*>(p + 256 + b_rows + b_s + b_k + up(b_out));
    RTB_CUDA_TRY(cudaMemsetAsync(err, 0, 256, s));
    if ((st = h2d(d_rows, rows, n_rows * row_len * sizeof(double), s)) != RTB_OK) return st;
    if ((st = h2d(d_s, qs.data(), qs.size() * sizeof(QeSurface), s)) != RTB_OK) return st;
    if ((st = h2d(d_k, knots.data(), knots.size() * sizeof(double), s)) != RTB_OK) return st;
    k_qe_curves<<<grid_for(total, 128, 16), 128, 0, s>>>(n_lambda, n_rows, d_rows, row_len, d_s, (int)qs.size(), d_k,
                                                          from_rows, d_l, d_q, err);
    if ((st = d2h(lambda, d_l, b_out, s)) != RTB_OK) return st;
    if ((st = d2h(qe, d_q, b_out, s)) != RTB_OK) return st;
    return finish(s, err, nullptr, nullptr);
}
