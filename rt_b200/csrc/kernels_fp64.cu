// kernels_fp64.cu -- plain FP64 kernels of the engine.
//
// Compiled with --fmad=false: every kernel here is bit-identical to the CPU
// oracle (see ray_fp64.cuh).  Three groups:
//   * drop-in kernels, one per engine call of common-lib/rt_engine_func.h;
//   * the per-surface trace kernel (one launch per surface, ray state in HBM);
//   * the fused FP64 trace kernel (whole scheme per ray, state in registers).
#include "trace_common.cuh"
#include "ray_fp64.cuh"
#include "philox.cuh"
#include "fused_fp64.cuh"

namespace rtb {

using f64::Ray;

// ===========================================================================
// Drop-in kernels
// ===========================================================================

__global__ void k_transform(size_t n, DevSurface s, double* X, double* Y, double* Z, double* cX, double* cY,
                            double* cZ) {
    for (size_t i = gtid(); i < n; i += gstride()) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        f64::transform(s, r);
        X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z; cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
}

__global__ void k_intersect(size_t n, DevSurface s, uint32_t fixes, double* X, double* Y, double* Z,
                            const double* cX, const double* cY, const double* cZ, char* flag,
                            unsigned long long* n_bad) {
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x; i0 < n; i0 += gstride()) {
        size_t i = i0 + threadIdx.x;
        bool lost = false;
        if (i < n) {
            Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
            lost = !f64::intersect(s, fixes, r);
            X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z;
            if (lost) flag[i] = 0;
        }
        warp_count(lost, n_bad);
    }
}

__global__ void k_reflect(size_t n, DevSurface s, const double* X, const double* Y, const double* Z, double* cX,
                          double* cY, double* cZ) {
    for (size_t i = gtid(); i < n; i += gstride()) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        f64::reflect(s, r);
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
}

// Refraction or diffraction (the action of a Lens or Grating surface).
__global__ void k_action(size_t n, DevSurface s, const double* knots, long long order, const double* lambda,
                         const double* X, const double* Y, const double* Z, double* cX, double* cY, double* cZ,
                         char* flag, unsigned long long* n_bad, unsigned* err) {
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x; i0 < n; i0 += gstride()) {
        size_t i = i0 + threadIdx.x;
        bool lost = false;
        if (i < n) {
            Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
            int a = f64::action(s, knots, order, lambda[i], r);
            if (a == f64::ACT_RANGE) {
                atomicOr(err, DEV_ERR_OUT_OF_RANGE);
            } else {
                lost = a == f64::ACT_LOST;
                cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
                if (lost) flag[i] = 0;
            }
        }
        warp_count(lost, n_bad);
    }
}

__global__ void k_normalize(size_t n, double* cX, double* cY, double* cZ) {
    for (size_t i = gtid(); i < n; i += gstride()) {
        double a = cX[i], b = cY[i], c = cZ[i];
        f64::normalize(a, b, c);
        cX[i] = a; cY[i] = b; cZ[i] = c;
    }
}

__global__ void k_aperture(size_t n, int shade, int shape, double sz0, double sz1, double c0, double c1,
                           const double* X, const double* Y, char* flag, unsigned long long* n_bad) {
    const double size[2] = {sz0, sz1}, center[2] = {c0, c1};
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x; i0 < n; i0 += gstride()) {
        size_t i = i0 + threadIdx.x;
        bool lost = false;
        if (i < n) {
            lost = !f64::aperture_pass(shade != 0, shape, size, center, X[i], Y[i]);
            if (lost) flag[i] = 0;
        }
        warp_count(lost, n_bad);
    }
}

__global__ void k_ccd_coords(size_t n, const double* X, const double* Y, double xsize, double ysize, double xpix,
                             double ypix, unsigned* ix, unsigned* iy) {
    for (size_t i = gtid(); i < n; i += gstride()) {
        unsigned a, b;
        ccd_coords(X[i], Y[i], xsize, ysize, xpix, ypix, a, b);
        ix[i] = a;
        iy[i] = b;
    }
}

// compute_ccd_image_kernel (rt_cuda_engine_ccd.cu:219-232, 280-288) with the
// spline evaluations on the device, a bounds check, and atomic accumulation.
__global__ void k_ccd_image(size_t n, const unsigned* ix, const unsigned* iy, const double* lambda,
                            const double* knots, int qe_off, int qe_n, int sp_off, int sp_n, size_t xdim, size_t ydim,
                            double pix_area, double* image, unsigned long long* n_outside, unsigned* err) {
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x; i0 < n; i0 += gstride()) {
        size_t i = i0 + threadIdx.x;
        bool outside = false;
        if (i < n) {
            double q, sp, l = lambda[i];
            if (!f64::table_eval(knots + qe_off, qe_n, l, q) || !f64::table_eval(knots + sp_off, sp_n, l, sp)) {
                atomicOr(err, DEV_ERR_OUT_OF_RANGE);
            } else {
                sp = sp * l;
                if (ix[i] >= xdim || iy[i] >= ydim) {
                    outside = true;
                } else {
                    unsigned index = iy[i] * (unsigned)xdim + ix[i];
                    atomicAdd(image + index, sp / K_HC * q * pix_area);
                }
            }
        }
        warp_count(outside, n_outside);
    }
}

__global__ void k_surface_qe(size_t n, const double* lambda, double* spec, const double* knots, int off, int cnt,
                             unsigned* err) {
    for (size_t i = gtid(); i < n; i += gstride()) {
        double q;
        if (!f64::table_eval(knots + off, cnt, lambda[i], q)) {
            atomicOr(err, DEV_ERR_OUT_OF_RANGE);
            continue;
        }
        spec[i] *= q;
    }
}

__global__ void k_beam_random(size_t n, double p1, double p2, double cx, double cy, double cz, uint64_t seed,
                              uint64_t first, double* X, double* Y, double* Z) {
    const double params[3] = {0.0, p1, p2}, center[3] = {cx, cy, cz};
    for (size_t i = gtid(); i < n; i += gstride()) {
        double u1, u2;
        ray_uniforms(seed, 0, first + i, u1, u2);
        disk_position(params, center, u1, u2, X[i], Y[i], Z[i]);
    }
}

__global__ void k_uniform_range(size_t n, double l0, double d_l, double* lambda) {
    for (size_t i = gtid(); i < n; i += gstride()) lambda[i] = l0 + (double)i * d_l;
}

__global__ void k_random_range(size_t n, double l0, double l1, uint64_t seed, double* lambda) {
    for (size_t i = gtid(); i < n; i += gstride()) {
        double u1, u2;
        ray_uniforms(seed, 1, i, u1, u2);
        lambda[i] = (l1 - l0) * u1 + l0;
    }
}

// rtb_generate_beams: disk positions, field-turned parallel cosines,
// composite wavelengths lambda_(i mod n_lambda).
__global__ void k_generate(const GenBeam* beams, int n_beams, uint64_t total, DevRays rays) {
    for (size_t i = gtid(); i < total; i += gstride()) {
        int lo = 0, hi = n_beams - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (beams[mid].first_ray <= i) lo = mid; else hi = mid - 1;
        }
        const GenBeam& b = beams[lo];
        uint64_t j = i - b.first_ray;
        if (j >= b.n_rays) continue;
        double u1, u2;
        ray_uniforms(b.seed, 0, j, u1, u2);
        disk_position(b.disk, b.center, u1, u2, rays.X[i], rays.Y[i], rays.Z[i]);
        rays.cX[i] = b.c0[0];
        rays.cY[i] = b.c0[1];
        rays.cZ[i] = b.c0[2];
        uint64_t k = j % b.n_lambda;
        rays.lambda[i] = (b.n_lambda == 1) ? b.range[0] : b.range[0] + (double)k * b.d_lambda;
        if (rays.flag) rays.flag[i] = 1;
        if (rays.lost_stage) rays.lost_stage[i] = RTB_NOT_LOST;
    }
}

// ===========================================================================
// Trace kernels
// ===========================================================================

// One surface of the per-surface engine.  Live rays (flag 1) are read, moved
// through the transform, Normalize, intersection, aperture, action and
// Normalize of surface k, and written back; a ray lost here gets
// lost_stage, flag 0 and the Normalize calls the reference would still
// apply to it.  After the last surface the survivors are counted.
// 64 registers: four 256-thread blocks per SM; the FP64 division and
// square-root chains need the warps more than the registers (measured on C1:
// 48 ms per pass at 64 registers, 67 ms at 98).
__global__ void __maxnreg__(64) k_surface_step(const DevScheme* __restrict__ sch, int k, const double* knots,
                                               const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                               unsigned long long* counts, unsigned* err) {
    const DevSurface& s = sch->s[k];
    const int n_stages = 3 * sch->n_surfaces;
    const bool last = k == sch->n_surfaces - 1;
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x; i0 < in.n; i0 += gstride()) {
        size_t i = i0 + threadIdx.x;
        bool ev = false;
        int key = 0;
        if (i < in.n && in.flag[i] == 1) {
            Ray r{in.X[i], in.Y[i], in.Z[i], in.cX[i], in.cY[i], in.cZ[i]};
            f64::transform(s, r);
            f64::normalize(r.cX, r.cY, r.cZ);
            int stage = -1;
            if (s.non_aux) {
                if (!f64::intersect(s, sch->fixes, r)) {
                    stage = 3 * k;
                } else if (!f64::aperture_pass(s.type == RTB_SHADE, s.shape, s.size, s.center, r.X, r.Y)) {
                    stage = 3 * k + 1;
                } else {
                    long long order = s.order;
                    if (s.type == RTB_GRATING) {
                        int b = beam_of(beams, n_beams, i);
                        if (beams[b].n_orders > 0) order = beams[b].orders[s.grating_index];
                    }
                    double lam = (s.type == RTB_LENS || s.type == RTB_GRATING) ? in.lambda[i] : 0.0;
                    int a = f64::action(s, knots, order, lam, r);
                    if (a == f64::ACT_RANGE) atomicOr(err, DEV_ERR_OUT_OF_RANGE);
                    else if (a == f64::ACT_LOST) stage = 3 * k + 2;
                    else f64::normalize(r.cX, r.cY, r.cZ);
                }
            }
            if (stage >= 0) {
                ev = true;
                if (sch->renorm_lost) f64::renormalize(r, s.renorm_after);
                out.flag[i] = 0;
                out.lost_stage[i] = (uint8_t)stage;
                key = beam_of(beams, n_beams, i) * (n_stages + 1) + stage;
            } else if (last) {
                ev = true;
                key = beam_of(beams, n_beams, i) * (n_stages + 1) + n_stages;
            }
            if (in.flag != out.flag) {
                if (stage < 0) out.flag[i] = 1;
                if (stage < 0) out.lost_stage[i] = RTB_NOT_LOST;
            }
            out.X[i] = r.X; out.Y[i] = r.Y; out.Z[i] = r.Z;
            out.cX[i] = r.cX; out.cY[i] = r.cY; out.cZ[i] = r.cZ;
        } else if (i < in.n && in.flag != out.flag) {
            out.flag[i] = in.flag[i];
        }
        count_event(ev, key, counts);
    }
}

// Frame counts over all good rays (rtb_ccd_frame).
__global__ void k_ccd_frame(DevRays rays, FrameArgs f) {
    for (size_t i0 = (size_t)blockIdx.x * blockDim.x; i0 < rays.n; i0 += gstride()) {
        size_t i = i0 + threadIdx.x;
        bool good = false;
        double X = 0, Y = 0;
        if (i < rays.n && rays.flag[i] == 1) {
            good = true;
            X = rays.X[i];
            Y = rays.Y[i];
        }
        frame_add(good, X, Y, f);
    }
}

// Fused FP64 trace for any scheme (fused_fp64.cuh); plans of a fixed scheme
// launch a copy specialised to it when one can be compiled (jit.cpp).
__global__ void __maxnreg__(64) k_fused_fp64(const DevScheme* __restrict__ g_sch, const double* knots,
                                             const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                             unsigned long long* counts, unsigned* err, int state_out,
                                             FrameArgs frame, TileSched ts) {
    fused_fp64<RtSurfacesF64>(g_sch, knots, beams, n_beams, in, out, counts, err, state_out, frame, ts);
}

}  // namespace rtb

namespace rtb {

// I1 of the blaze function after Tarasov (rt_cuda_engine_surface.cu:1988-2019):
// blaze angle c, incidence k1 (alpha), grating constant eps, relative rule
// length rule_size.
__device__ __forceinline__ double i1_tarasov(double c, double k1, double eps, double rule_size, double lambda,
                                             double beta) {
    double I1 = K_RT_PI * eps * rule_size / lambda * cos(beta) / cos(c - beta) * (sin(c - k1) + sin(c - beta));
    double term = cos(beta) * cos(c - k1) / cos(c - beta);
    if (fabs(I1) < K_RT_PI / 2.0) {
        I1 *= I1;
        I1 = (0.00761 * I1 - 0.16605) * I1 + 1;
    } else {
        I1 = sin(I1) / (I1);
    }
    I1 *= term;
    I1 *= I1;
    return I1;
}

// grating_energy_distr_kernel (rt_cuda_engine_surface.cu:2098-2153) for one
// wavelength: the energy in `order`, normalised over all propagating orders.
__device__ __forceinline__ double grating_energy(double l, long long order, double blaze, double alpha, double gamma,
                                                 double gr_const, double rule_size) {
    double sin_alpha = sin(alpha);
    double cos_gamma = cos(gamma);
    long long order_min = __double2ll_rz(gr_const / l * (sin_alpha - 1) * cos_gamma);
    long long order_max = __double2ll_rz(gr_const / l * (sin_alpha + 1) * cos_gamma);
    double norm = 0.0;
    for (long long m = order_min; m <= order_max; ++m) {
        double beta = asin(m * l / gr_const / cos_gamma - sin_alpha);
        norm += i1_tarasov(blaze, alpha, gr_const, rule_size, l, beta);
    }
    double beta = asin(order * l / (gr_const * cos_gamma) - sin_alpha);
    double I1 = i1_tarasov(blaze, alpha, gr_const, rule_size, l, beta);
    return I1 / norm;
}

__global__ void k_grating_energy(size_t n, const double* lambda, long long order, double blaze, double alpha,
                                 double gamma, double gr_const, double rule_start, double rule_stop, double* energy) {
    const double rule_size = rule_stop - rule_start;
    for (size_t i = gtid(); i < n; i += gstride())
        energy[i] *= grating_energy(lambda[i], order, blaze, alpha, gamma, gr_const, rule_size);
}

// Scheme::ComputeQE's curves (scheme.cpp:1249-1316), every range in one
// launch: element e = r * n_lambda + i is wavelength i of range r,
// lambda = w1 + (w2 - w1) / (n_lambda - 1) * i, and its throughput is 1
// multiplied, surface after surface, by QE(lambda) (surface_QE) and, for a
// grating, by its energy in |order| (grating_energy_distr): the products in
// the order the reference's per-surface calls make them.  With more than one
// range, grating g takes its order from column 2 + g of the range row.
__global__ void k_qe_curves(size_t n_lambda, size_t n_rows, const double* rows, size_t row_len, const QeSurface* s,
                            int n_s, const double* knots, int orders_from_rows, double* lambda, double* qe,
                            unsigned* err) {
    const size_t total = n_lambda * n_rows;
    for (size_t e = gtid(); e < total; e += gstride()) {
        const size_t r = e / n_lambda, i = e - r * n_lambda;
        const double* row = rows + r * row_len;
        const double d_lambda = (row[1] - row[0]) / (double)(n_lambda - 1);
        const double l = row[0] + d_lambda * (double)i;
        double q = 1.0;
        int g = 0;
        for (int k = 0; k < n_s; ++k) {
            double v;
            if (!f64::table_eval(knots + s[k].off, s[k].cnt, l, v)) {
                atomicOr(err, DEV_ERR_OUT_OF_RANGE);
                break;
            }
            q *= v;
            if (s[k].grating) {
                long long order = orders_from_rows ? (long long)(long)row[2 + g] : s[k].order;
                ++g;
                if (order < 0) order = -order;
                q *= grating_energy(l, order, s[k].blaze, s[k].alpha, s[k].gamma, s[k].gr_const, s[k].rule_size);
            }
        }
        lambda[e] = l;
        qe[e] = q;
    }
}

}  // namespace rtb
