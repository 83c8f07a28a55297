// mixed32.cuh -- device code of the FP32-state fused trace kernel
// (RTB_MIXED32).
//
// The ray state is FP32: the position on the last surface met, in that
// surface's frame (relative to the beam's origin before the first), and the
// direction cosines.  The bulk of the per-ray arithmetic runs in FP32 on it:
// the transforms (one 3x3 rotation per surface, any Aux surfaces before it
// folded in on the host), the surface normals, reflection, refraction and
// the renormalisation of the cosines, with MUFU reciprocals and square
// roots.  FP64 is kept where it sets the CCD position to well below the
// 0.05 um budget:
//   * the intersection root: the ray's start in the new frame is the FP32
//     rotated position plus the FP64 vertex offset, and the roots of
//     mixed.cuh (cancellation-safe conic quadratic, Newton on the even
//     asphere and the toric, stopping after a step below 1e-5 mm with the
//     root good to ~1e-12 mm) run in FP64 on it; the aperture test runs on the
//     FP64 point before it is rounded to the FP32 state;
//   * the grating equation (mx::diffract);
//   * the detector coordinate: the last surface's FP64 intersection point
//     is the output.
// The refractive indices come from the FP64 table evaluation of mixed.cuh
// (once per ray for a lens's two surfaces); their ratio is rounded to FP32
// for the refraction.  Accuracy is measured against the FP64 oracle (median,
// p99.9 and max CCD error in um).
#pragma once

#include "mixed.cuh"
#include "rowpipe.cuh"

namespace rtb {
namespace m32 {

struct Ray {
    float X, Y, Z, cX, cY, cZ;
};

__device__ __forceinline__ float rcp(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float rsqrt(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sqrt(x): x * rsqrt(x) with one Newton correction of the product; NaN for
// x < 0, 0 for x == 0.
__device__ __forceinline__ float sqrt_(float x) {
    if (!(x > 0.0f)) return (x == 0.0f) ? 0.0f : __int_as_float(0x7fc00000);
    const float y = rsqrt(x);
    const float s = x * y;
    return fmaf(0.5f * y, fmaf(-s, s, x), s);
}

// Unit direction: rsqrt seed and one Newton step (error ~1 ulp).
__device__ __forceinline__ void normalize(Ray& r) {
    const float s = fmaf(r.cX, r.cX, fmaf(r.cY, r.cY, r.cZ * r.cZ));
    float k = rsqrt(s);
    k = k * fmaf(-0.5f * s * k, k, 1.5f);
    r.cX *= k;
    r.cY *= k;
    r.cZ *= k;
}

// Paired FP32 arithmetic of sm_100 (FFMA2 / FMUL2): one instruction computes
// two independent single-precision results, each rounded as fmaf / __fmul_rn
// would round it.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// P <- M P and D <- M D together, M given by rows as (m, m) pairs: the
// position and the direction cosine along each axis form one pair, so the
// two rotations take nine paired instructions instead of eighteen.
__device__ __forceinline__ void rotate(const float2* m, Ray& r) {
    const float2 x = make_float2(r.X, r.cX), y = make_float2(r.Y, r.cY), z = make_float2(r.Z, r.cZ);
    const float2 a = fma2(m[0], x, fma2(m[1], y, mul2(m[2], z)));
    const float2 b = fma2(m[3], x, fma2(m[4], y, mul2(m[5], z)));
    const float2 c = fma2(m[6], x, fma2(m[7], y, mul2(m[8], z)));
    r.X = a.x;
    r.cX = a.y;
    r.Y = b.x;
    r.cY = b.y;
    r.Z = c.x;
    r.cZ = c.y;
}

// (dF/dX, dF/dY) of the conic + even polynomial (conic_derivs,
// rt_cuda_engine_surface.cu:45-61); dF/dZ = 1.
template <class Sh>
__device__ __forceinline__ void conic_normal(const DevSurface& s, float x, float y, float& nx, float& ny) {
    const float r2 = fmaf(x, x, y * y);
    const float c = s.f_c, k1 = s.f_k1;
    float E = c * rsqrt(fmaf(-k1 * c * c, r2, 1.0f));
    float sum = 0.0f, rr = 1.0f;
    const int N = Sh::n_poly(s);
    for (int i = 1; i <= N; ++i, rr *= r2) sum = fmaf(s.f_ipoly[i - 1], rr, sum);
    E = fmaf(2.0f, sum, E);
    nx = -E * x;
    ny = -E * y;
}

// (dF/dX, dF/dY, dF/dZ) of the toric surface (toric_derivs, surface.cu:65-94).
template <class Sh>
__device__ __forceinline__ void toric_normal(const DevSurface& s, float x, float y, float z, float& nx, float& ny,
                                             float& nz) {
    const float Y2 = y * y;
    const float c = s.f_c, k1 = s.f_k1, cR = s.f_cR;
    const float q = fmaf(-k1 * c * c, Y2, 1.0f);
    const float rq = rsqrt(q);
    float Fy = c * Y2 * rcp(1.0f + q * rq);
    float sum = 0.0f, rr = Y2;
    const int N = Sh::n_poly(s);
    for (int i = 0; i < N; ++i, rr *= Y2) sum = fmaf(s.f_poly[i], rr, sum);
    Fy += sum;
    float dFy = c * y * rq;
    sum = 0.0f;
    rr = 1.0f;
    for (int i = 1; i <= N; ++i, rr *= Y2) sum = fmaf(s.f_ipoly[i - 1], rr, sum);
    dFy = fmaf(2.0f, sum, dFy);
    nx = -cR * x;
    ny = (cR * Fy - 1.0f) * dFy;
    nz = fmaf(-cR, z, 1.0f);
}

template <class Sh>
__device__ __forceinline__ void normal(const DevSurface& s, const Ray& r, float& nx, float& ny, float& nz) {
    if (Sh::cls(s) == RTB_TORIC) {
        toric_normal<Sh>(s, r.X, r.Y, r.Z, nx, ny, nz);
    } else {
        conic_normal<Sh>(s, r.X, r.Y, nx, ny);
        nz = 1.0f;
    }
}

// k' = k - 2 (k.N) N / |N|^2 (surface.cu:771-827).
__device__ __forceinline__ void reflect(float nx, float ny, float nz, Ray& r) {
    const float a2 = 2.0f * fmaf(r.cX, nx, fmaf(r.cY, ny, r.cZ * nz)) * rcp(fmaf(nx, nx, fmaf(ny, ny, nz * nz)));
    r.cX = fmaf(-a2, nx, r.cX);
    r.cY = fmaf(-a2, ny, r.cY);
    r.cZ = fmaf(-a2, nz, r.cZ);
}

// Vector Snell law (surface.cu:956-1066): false on total internal reflection.
__device__ __forceinline__ bool refract(float mu, float nx, float ny, float nz, Ray& r) {
    const float iG = rcp(fmaf(nx, nx, fmaf(ny, ny, nz * nz)));
    const float a = mu * fmaf(r.cX, nx, fmaf(r.cY, ny, r.cZ * nz)) * iG;
    const float b = fmaf(mu, mu, -1.0f) * iG;
    const float a2 = a * a;
    if (b > a2) return false;
    const float G = -a + sqrt_(a2 - b);
    r.cX = fmaf(mu, r.cX, G * nx);
    r.cY = fmaf(mu, r.cY, G * ny);
    r.cZ = fmaf(mu, r.cZ, G * nz);
    return true;
}

}  // namespace m32

// One surface of the FP32-state engine on one ray: -1 survived, a stage >= 0
// that lost it, -2 a wavelength outside a table.  q holds the ray's FP64
// point on this surface afterwards (the detector coordinate after the last
// surface; the point where it was lost otherwise).
template <class Sh = RtShape>
__device__ __forceinline__ int m32_surface(const DevSurface& s, int k, uint32_t fixes, const double* knots,
                                           const BeamCtx& bc, const double* off0, double lam,
                                           mx::TableMemo& memo, m32::Ray& r, mx::Ray& q) {
    if (!Sh::non_aux(s)) return -1;  // its transform is folded into the next surface's
    if (Sh::rot32(s)) m32::rotate(s.m32, r);
    const double* off = Sh::first32(s) ? off0 : s.off32;
    q = mx::Ray{(double)r.X + off[0], (double)r.Y + off[1], (double)r.Z + off[2],
                (double)r.cX,         (double)r.cY,         (double)r.cZ};
    const int hit = mx::intersect<Sh>(s, fixes, q);
    if (hit == 1) return 3 * k;
    if (hit == 2) return 3 * k + 1;
    if (!f64::aperture_pass(Sh::type(s) == RTB_SHADE, Sh::shape(s), s.size, s.center, q.X, q.Y)) return 3 * k + 1;
    r.X = (float)q.X;
    r.Y = (float)q.Y;
    r.Z = (float)q.Z;
    const int type = Sh::type(s), cls = Sh::cls(s), gr_type = Sh::gr_type(s);
    if (type == RTB_MIRROR) {
        if (cls == RTB_PLANE) {
            r.cZ = -r.cZ;
        } else {
            float nx, ny, nz;
            m32::normal<Sh>(s, r, nx, ny, nz);
            m32::reflect(nx, ny, nz, r);
            m32::normalize(r);
        }
        return -1;
    }
    if (type != RTB_LENS && type != RTB_GRATING) return -1;
    double n1v = 1.0, n2v = 1.0;
    {
        const int first = (type == RTB_LENS || gr_type == RTB_TRANSPARENT) ? 0 : 1;
#pragma unroll 1
        for (int t = first; t < 2; ++t) {
            double v;
            if (!mx::table_at(knots, t ? s.n2_off : s.n1_off, t ? s.n2_n : s.n1_n, t ? s.n2_invh : s.n1_invh, lam,
                              memo, v))
                return -2;
            if (t) n2v = v;
            else n1v = v;
        }
    }
    float nx = 0.0f, ny = 0.0f, nz = 1.0f;
    if (cls != RTB_PLANE) m32::normal<Sh>(s, r, nx, ny, nz);
    const double in2 = mx::rcp(n2v);
    if (type == RTB_LENS) {
        if (!m32::refract((float)(n1v * in2), nx, ny, nz, r)) return 3 * k + 2;
        m32::normalize(r);
        return -1;
    }
    // the grating equation in FP64 on the FP64 cosines
    const long long order = bc.order(s);
    const double mu = (gr_type == RTB_TRANSPARENT) ? n1v * in2 : 0.0;
    const double L = (double)order * lam * in2 * s.inv_gr;
    if (!mx::diffract<Sh>(s, mu, L, (double)nx, (double)ny, (double)nz, q)) return 3 * k + 2;
    if (cls == RTB_TORIC) mx::normalize(q);  // the toric rule direction leaves the cosines off unit length
    r.cX = (float)q.cX;
    r.cY = (float)q.cY;
    r.cZ = (float)q.cZ;
    return -1;
}

// The surfaces of one ray in order, until one loses it (RtShape: each
// surface's structure read from the scheme; jit.cpp writes the same with a
// FixedShape per surface).
struct Rt32Surfaces {
    __device__ __forceinline__ static void run(const DevScheme* sch, const double* knots, const BeamCtx& bc,
                                               const double* off0, double lam, mx::TableMemo& memo, m32::Ray& r,
                                               mx::Ray& q, int& stage) {
        for (int k = 0; k < sch->n_surfaces && stage == -1; ++k)
            stage = m32_surface(sch->s[k], k, sch->fixes, knots, bc, off0, lam, memo, r, q);
    }
};

// Fused FP32-state trace: the persistent row loop of fused_mixed with the
// FP32 state.  Plans feed it Row32 blocks (positions relative to the beam's
// origin) through the row pipeline; one-shot traces feed it the FP64 arrays,
// converted on load.
template <class Surfaces>
__device__ __forceinline__ void fused_mixed32(const DevScheme* __restrict__ g_sch, const double* knots,
                                              const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                              unsigned long long* counts, unsigned* err, int state_out,
                                              FrameArgs frame, TileSched ts) {
    const double* s_knots;
    const DevScheme* sch = stage_scheme(g_sch, knots, s_knots);
    const int n_stages = 3 * sch->n_surfaces;
    RowLoop rows(ts, in.n, warp_row_buffer<Row32>(sch->n_knots), (unsigned)sizeof(Row32), err);
    const int lane = threadIdx.x & 31;
    BeamCursor cur;
    while (rows.begin()) {
        const size_t slot = rows.slot();
        const bool valid = slot < in.n;
        // the ray's index, read only when its results go there; its beam: the
        // beam of its slot in a plan's (beam-major) tracing order
        const size_t i = (ts.order && valid && !(rows.packed && ts.out_by_slot)) ? (size_t)ts.order[slot] : slot;
        const size_t oi = ts.out_by_slot ? slot : i;
        const size_t bi = rows.packed ? slot : i;
        const int b = valid ? cur.at(beams, n_beams, bi) : 0;
        m32::Ray r{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        double lam = 0.0;
        char f = 0;
        if (rows.packed) {
            const Row32& w = rows.row<Row32>();
            f = w.flag[lane];
            r = m32::Ray{w.X[lane], w.Y[lane], w.Z[lane], w.cX[lane], w.cY[lane], w.cZ[lane]};
            lam = w.lambda[lane];
        } else if (valid) {
            const size_t ri = ts.in_by_slot ? slot : i;
            f = in.flag[ri];
            if (f == 1) {
                const DevBeam& bm = beams[b];
                r = m32::Ray{(float)(in.X[ri] - bm.origin[0]), (float)(in.Y[ri] - bm.origin[1]),
                             (float)(in.Z[ri] - bm.origin[2]), (float)in.cX[ri], (float)in.cY[ri],
                             (float)in.cZ[ri]};
                lam = in.lambda[ri];
            }
        }
        rows.prefetch();
        bool ev = false, good = false;
        int key = 0;
        double outX = 0, outY = 0;
        if (valid && f == 1) {
            const BeamCtx& bc = cur.ctx;
            const double off0[3] = {bc.bm->off0[0], bc.bm->off0[1], bc.bm->off0[2]};
            if (!rows.packed) m32::normalize(r);  // row blocks hold normalised cosines
            mx::TableMemo memo;
            mx::Ray q{0, 0, 0, 0, 0, 0};
            int stage = -1;
            Surfaces::run(sch, s_knots, bc, off0, lam, memo, r, q, stage);
            if (stage == -1 && sch->tail_on) {  // Aux surfaces after the last one, in FP64
                const double* m = sch->tail_m;
                const double* o = sch->tail_off;
                const double x = q.X, y = q.Y, z = q.Z, cx = r.cX, cy = r.cY, cz = r.cZ;
                q.X = fma(m[0], x, fma(m[1], y, fma(m[2], z, o[0])));
                q.Y = fma(m[3], x, fma(m[4], y, fma(m[5], z, o[1])));
                q.Z = fma(m[6], x, fma(m[7], y, fma(m[8], z, o[2])));
                r.cX = (float)fma(m[0], cx, fma(m[1], cy, m[2] * cz));
                r.cY = (float)fma(m[3], cx, fma(m[4], cy, m[5] * cz));
                r.cZ = (float)fma(m[6], cx, fma(m[7], cy, m[8] * cz));
            }
            if (stage == -2) atomicOr(err, DEV_ERR_OUT_OF_RANGE);
            if (stage >= 0) {
                ev = true;
                out.flag[oi] = 0;
                out.lost_stage[oi] = (uint8_t)stage;
                key = b * (n_stages + 1) + stage;
            } else if (stage == -1) {
                ev = good = true;
                key = b * (n_stages + 1) + n_stages;
                if (rows.packed || in.flag != out.flag) {
                    out.flag[oi] = 1;
                    out.lost_stage[oi] = RTB_NOT_LOST;
                }
            }
            if (stage != -2) {
                out.X[oi] = q.X;
                out.Y[oi] = q.Y;
                if (state_out) {
                    out.Z[oi] = q.Z;
                    out.cX[oi] = r.cX;
                    out.cY[oi] = r.cY;
                    out.cZ[oi] = r.cZ;
                }
            }
            outX = q.X;
            outY = q.Y;
        } else if (valid && (rows.packed || in.flag != out.flag)) {
            out.flag[oi] = f;
        }
        count_event(ev, key, counts);
        if (frame.counts) frame_add<false>(good, outX, outY, frame);
    }
}

}  // namespace rtb
