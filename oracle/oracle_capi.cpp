// oracle_capi.cpp -- C entry points of the CPU oracle (liboracle.so).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
// bench.py's CPU baseline through ctypes; never by the product.  Function
// names are the product's rtb_* names with an oracle_ prefix and the same
// arguments, so a test can run one call against both and compare.
//
// Two formulations of the per-surface loop of Scheme::run
// (common-lib/scheme.cpp:983-1055) are provided:
//   * oracle_trace: ray by ray, rays keep their index, lost rays carry the
//     stage that lost them (what the B200 engine computes);
//   * oracle_trace_literal: array by array with the reference's Rearrange
//     after each lossy stage and Normalize over all rays, statement for
//     statement as the reference host loop runs it.
// Tests check that the two agree once oracle_reference_order permutes the
// first one.
#include "rt_oracle.hpp"
#include "flop_count.hpp"
#include "../include/rtb.h"

#include <atomic>
#include <vector>
#include <cstdio>

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace rto;

namespace {

struct Prepared {
    int cls, type, shape, gr_type;
    long order;
    double gr_const;
    SurfConst sc;
    IsectKind kind;
    TransformConst tc;
    double size[2], center[2];
    rtb_table n1, n2;
    int grating_index;     // position among gratings, -1 otherwise
    bool non_aux;
    int renorm_after;      // Normalize calls after this surface's action (for lost rays)
    int surfaces_upto;     // non-Aux surfaces up to and including this one
};

int prepare(const rtb_surface* s, size_t n, std::vector<Prepared>& out) {
    if (n == 0 || n > RTB_MAX_SURFACES) return BAD_VALUE;
    out.resize(n);
    int ng = 0, nonaux = 0;
    for (size_t k = 0; k < n; ++k) {
        Prepared& p = out[k];
        p.cls = s[k].cls; p.type = s[k].type; p.shape = s[k].shape; p.gr_type = s[k].grating_type;
        p.order = (long)s[k].order; p.gr_const = s[k].gr_const;
        p.non_aux = s[k].type != AuxType;
        if (p.non_aux) {
            Status st = make_surf_const(p.cls, s[k].params, p.sc);
            if (st != OK) return st;
            p.kind = intersection_kind(p.cls, s[k].params);
        } else {
            p.kind = IS_NONE;
        }
        double ang[3];
        for (int i = 0; i < 3; ++i) ang[i] = scheme_angle_rad(s[k].angles_deg[i]);
        p.tc = make_transform(ang, s[k].distance);
        for (int i = 0; i < 2; ++i) { p.size[i] = s[k].size[i]; p.center[i] = s[k].center[i]; }
        p.n1 = s[k].n1; p.n2 = s[k].n2;
        p.grating_index = (p.type == Grating) ? ng++ : -1;
        if (p.non_aux) ++nonaux;
        p.surfaces_upto = nonaux;
    }
    if (ng > RTB_MAX_GRATINGS) return BAD_VALUE;
    for (size_t k = 0; k < n; ++k) {
        int cnt = out[k].non_aux ? 1 : 0;   // the Normalize after this surface's action
        for (size_t j = k + 1; j < n; ++j) cnt += 1 + (out[j].non_aux ? 1 : 0);
        out[k].renorm_after = cnt;
    }
    return OK;
}

template <class T>
inline bool eval_table(const rtb_table& t, T x, T& v) {
    return table_eval(t.n, t.x, t.y, t.y2, x, v);
}

// Normalize a lost ray `count` times; stops at the fixed point.
template <class T>
inline void renormalize(RayT<T>& r, int count) {
    for (int i = 0; i < count; ++i) {
        T a = r.cX, b = r.cY, c = r.cZ;
        normalize(a, b, c);
        if (a == r.cX && b == r.cY && c == r.cZ) break;
        r.cX = a; r.cY = b; r.cZ = c;
    }
}

// Action of a surface on one ray (Mirror/Lens/Grating ::Action,
// surface.cpp:385-396,453-472,563-585).  Returns OK, OUT_OF_RANGE, or
// NO_GOOD_RAYS meaning "this ray is lost".
template <class T>
inline int action(const Prepared& p, const SurfConstT<T>& sc, const long* orders, int n_orders, T lambda,
                  RayT<T>& r) {
    switch (p.type) {
        case Mirror: reflect(p.cls, sc, r); return OK;
        case Lens: {
            T a, b;
            if (!eval_table(p.n1, lambda, a) || !eval_table(p.n2, lambda, b)) return OUT_OF_RANGE;
            T mu = a;
            mu /= b;
            return refract(p.cls, sc, mu, r) ? OK : NO_GOOD_RAYS;
        }
        case Grating: {
            long ord = (n_orders > 0) ? orders[p.grating_index] : p.order;
            T n2v, mu = 0.0;
            if (!eval_table(p.n2, lambda, n2v)) return OUT_OF_RANGE;
            if (p.gr_type == Transparent) {
                T n1v;
                if (!eval_table(p.n1, lambda, n1v)) return OUT_OF_RANGE;
                mu = n1v;
                mu /= n2v;
            } else if (p.gr_type != Reflective) {
                return BAD_VALUE;
            }
            T L = T((double)ord) * lambda / n2v / p.gr_const;
            return diffract(p.cls, p.gr_type, sc, mu, L, r) ? OK : NO_GOOD_RAYS;
        }
        default: return OK;
    }
}

// Trace one ray through all surfaces.  Returns a status; sets lost_stage.
// `at(k)` is called as the ray enters surface k and, with k = S.size(),
// after its last one (the operation counter attributes by it).
template <class T, class At>
inline int trace_ray(const std::vector<Prepared>& S, const SurfConstT<T>* SC, const long* orders, int n_orders,
                     T lambda, int renorm_lost, uint32_t fixes, RayT<T>& r, int& lost_stage, At&& at) {
    lost_stage = RTB_NOT_LOST;
    for (size_t k = 0; k < S.size(); ++k) {
        const Prepared& p = S[k];
        at(k);
        transform(p.tc, r);
        normalize(r.cX, r.cY, r.cZ);
        if (!p.non_aux) continue;
        int stage = (int)(3 * k);
        if (!intersect(p.kind, SC[k], fixes, r)) { lost_stage = stage; break; }
        bool shade = p.type == Shade;
        if (!aperture_pass(shade, p.shape, p.size, p.center, r.X, r.Y)) { lost_stage = stage + 1; break; }
        int st = action(p, SC[k], orders, n_orders, lambda, r);
        if (st == NO_GOOD_RAYS) { lost_stage = stage + 2; break; }
        if (st != OK) return st;
        normalize(r.cX, r.cY, r.cZ);
    }
    at(S.size());
    if (lost_stage != RTB_NOT_LOST && renorm_lost) renormalize(r, S[lost_stage / 3].renorm_after);
    return OK;
}

inline std::vector<SurfConst> surface_constants(const std::vector<Prepared>& S) {
    std::vector<SurfConst> sc(S.size());
    for (size_t k = 0; k < S.size(); ++k) sc[k] = S[k].sc;
    return sc;
}

}  // namespace

extern "C" {

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// ---- beam generation ------------------------------------------------------

void oracle_beam_sincos(size_t n, const double* x, double* s, double* c) {
    for (size_t i = 0; i < n; ++i) beam_sincos(x[i], s[i], c[i]);
}

void oracle_philox(size_t n, uint64_t seed, uint64_t stream, uint64_t first, double* u1, double* u2) {
    for (size_t i = 0; i < n; ++i) ray_uniforms(seed, stream, first + i, u1[i], u2[i]);
}

// rtb_beam_random on the CPU.
int oracle_beam_random(int shape, const double* params, const double* center, size_t n,
                       double* X, double* Y, double* Z, uint64_t seed, uint64_t first_ray) {
    if (shape != Circle) return BAD_VALUE;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        double u1, u2;
        ray_uniforms(seed, 0, first_ray + (uint64_t)i, u1, u2);
        disk_position(params, center, u1, u2, X[i], Y[i], Z[i]);
    }
    return OK;
}

int oracle_uniform_range_beam(size_t n, const double* range, double* lambda) {
    for (size_t j = 0; j < n; ++j) lambda[j] = uniform_lambda(range, n, j);
    return OK;
}

// rtb_generate_beams on the CPU (host arrays).
int oracle_generate_beams(const rtb_beam* beams, size_t n_beams, const rtb_rays* rays) {
    for (size_t b = 0; b < n_beams; ++b) {
        const rtb_beam& bm = beams[b];
        if (bm.first_ray + bm.n_rays > rays->n || bm.n_lambda == 0) return BAD_VALUE;
        double tx = std::tan(bm.field[0]), ty = std::tan(bm.field[1]);
        double cx0 = tx, cy0 = ty, cz0 = 1.0;
        normalize(cx0, cy0, cz0);
        std::vector<double> lam(bm.n_lambda);
        if (bm.n_lambda == 1) lam[0] = bm.range[0];
        else for (size_t j = 0; j < bm.n_lambda; ++j) lam[j] = uniform_lambda(bm.range, bm.n_lambda, j);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)bm.n_rays; ++i) {
            size_t k = bm.first_ray + (size_t)i;
            double u1, u2;
            ray_uniforms(bm.seed, 0, (uint64_t)i, u1, u2);
            disk_position(bm.disk, bm.center, u1, u2, rays->X[k], rays->Y[k], rays->Z[k]);
            rays->cX[k] = cx0; rays->cY[k] = cy0; rays->cZ[k] = cz0;
            rays->lambda[k] = lam[(size_t)i % bm.n_lambda];
            if (rays->flag) rays->flag[k] = 1;
            if (rays->lost_stage) rays->lost_stage[k] = RTB_NOT_LOST;
        }
    }
    return OK;
}

// ---- per-call functions (same arguments as the rtb_* drop-in calls) ------

int oracle_beam_transform(size_t n, const double* angles, const double* dist,
                          double* X, double* Y, double* Z, double* cX, double* cY, double* cZ) {
    TransformConst t = make_transform(angles, dist);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        transform(t, r);
        X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z; cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    return OK;
}

int oracle_surface_intersection_fix(int cls, const double* params, size_t n, double* X, double* Y,
                                    double* Z, double* cX, double* cY, double* cZ, size_t* n_bad,
                                    char* flag, uint32_t fixes) {
    SurfConst s;
    if (cls == Plane || cls == Conic || cls == Toric) {
        if (make_surf_const(cls, params, s) != OK) return BAD_VALUE;
    } else {
        return OK;  // AUX: nothing (surface.cu:634-635)
    }
    IsectKind kind = intersection_kind(cls, params);
    size_t bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (long long i = 0; i < (long long)n; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        if (!intersect(kind, s, fixes, r)) { flag[i] = 0; ++bad; }
        X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z;
    }
    *n_bad += bad;
    return OK;
}

int oracle_surface_intersection(int cls, const double* params, size_t n, double* X, double* Y,
                                double* Z, double* cX, double* cY, double* cZ, size_t* n_bad, char* flag) {
    return oracle_surface_intersection_fix(cls, params, n, X, Y, Z, cX, cY, cZ, n_bad, flag, 0);
}

int oracle_surface_reflection(int cls, const double* params, size_t n, double* X, double* Y, double* Z,
                              double* cX, double* cY, double* cZ) {
    SurfConst s;
    if (make_surf_const(cls, params, s) != OK) return BAD_VALUE;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        reflect(cls, s, r);
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    return OK;
}

int oracle_surface_refraction(int cls, const double* params, size_t n, double* X, double* Y, double* Z,
                              double* cX, double* cY, double* cZ, const double* lambda,
                              const rtb_table* n1, const rtb_table* n2, size_t* n_bad, char* flag) {
    SurfConst s;
    if (make_surf_const(cls, params, s) != OK) return BAD_VALUE;
    size_t bad = 0;
    std::atomic<int> err{0};
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (long long i = 0; i < (long long)n; ++i) {
        double a, b;
        if (!eval_table(*n1, lambda[i], a) || !eval_table(*n2, lambda[i], b)) { err = OUT_OF_RANGE; continue; }
        double mu = a;
        mu /= b;
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        if (!refract(cls, s, mu, r)) { flag[i] = 0; ++bad; }
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    if (err) return err;
    *n_bad += bad;
    return OK;
}

int oracle_surface_diffration(int cls, int gr_type, const double* params, long diff_order,
                              double gr_constant, size_t n, double* X, double* Y, double* Z,
                              double* cX, double* cY, double* cZ, const double* lambda,
                              const rtb_table* n1, const rtb_table* n2, size_t* n_bad, char* flag) {
    SurfConst s;
    if (make_surf_const(cls, params, s) != OK) return BAD_VALUE;
    if (gr_type != Reflective && gr_type != Transparent) return BAD_VALUE;
    size_t bad = 0;
    std::atomic<int> err{0};
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (long long i = 0; i < (long long)n; ++i) {
        double n2v, mu = 0.0;
        if (!eval_table(*n2, lambda[i], n2v)) { err = OUT_OF_RANGE; continue; }
        if (gr_type == Transparent) {
            double n1v;
            if (!eval_table(*n1, lambda[i], n1v)) { err = OUT_OF_RANGE; continue; }
            mu = n1v;
            mu /= n2v;
        }
        double L = diff_order * lambda[i] / n2v / gr_constant;
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        if (!diffract(cls, gr_type, s, mu, L, r)) { flag[i] = 0; ++bad; }
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    if (err) return err;
    *n_bad += bad;
    return OK;
}

int oracle_spline_init(size_t n, const double* x, const double* y, double* y2) {
    if (n < 4) return BAD_VALUE;
    spline_init(n, x, y, y2);
    return OK;
}

int oracle_table_eval(const rtb_table* t, size_t n, const double* xs, double* out) {
    for (size_t i = 0; i < n; ++i)
        if (!eval_table(*t, xs[i], out[i])) return OUT_OF_RANGE;
    return OK;
}

int oracle_normalize(size_t n, double* cX, double* cY, double* cZ) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) normalize(cX[i], cY[i], cZ[i]);
    return OK;
}

int oracle_apply_constrains(int shade, int shape, const double* size, const double* center, size_t n,
                            const double* X, const double* Y, char* flag, size_t* n_bad) {
    size_t bad = 0;
    for (size_t i = 0; i < n; ++i)
        if (!aperture_pass(shade != 0, shape, size, center, X[i], Y[i])) { flag[i] = 0; ++bad; }
    *n_bad += bad;
    return OK;
}

int oracle_rearrange(size_t* n_good, double* X, double* Y, double* Z, double* cX, double* cY,
                     double* cZ, double* lambda, char* flag) {
    double* arr[7] = {X, Y, Z, cX, cY, cZ, lambda};
    *n_good = rearrange(flag, *n_good, [&](size_t a, size_t b) {
        for (double* v : arr) std::swap(v[a], v[b]);
    });
    return OK;
}

int oracle_ccd_coordinates(size_t n, const double* X, const double* Y, double xsize, double ysize,
                           double xpix, double ypix, unsigned int* ix, unsigned int* iy) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t a, b;
        ccd_coords(X[i], Y[i], xsize, ysize, xpix, ypix, a, b);
        ix[i] = a; iy[i] = b;
    }
    return OK;
}

// compute_ccd_image (ccd.cu:219-232,280-288,360) with a bounds check; rays
// are added in index order.
int oracle_compute_ccd_image(size_t n, const unsigned int* ix, const unsigned int* iy,
                             const double* lambda, const rtb_table* qe, const rtb_table* spec,
                             size_t xdim, size_t ydim, double xpix, double ypix, double* image,
                             uint64_t* n_outside) {
    double pix_area = xpix * ypix * 1.0E-2;
    uint64_t outside = 0;
    for (size_t i = 0; i < n; ++i) {
        double q, sp;
        if (!eval_table(*qe, lambda[i], q) || !eval_table(*spec, lambda[i], sp)) return OUT_OF_RANGE;
        sp = sp * lambda[i];
        if (ix[i] >= xdim || iy[i] >= ydim) { ++outside; continue; }
        unsigned int index = iy[i] * (unsigned int)xdim + ix[i];
        image[index] += sp / HC * q * pix_area;
    }
    if (n_outside) *n_outside += outside;
    return OK;
}

int oracle_surface_QE(size_t n, const double* lambda, double* spec, const rtb_table* qe) {
    for (size_t i = 0; i < n; ++i) {
        double q;
        if (!eval_table(*qe, lambda[i], q)) return OUT_OF_RANGE;
        spec[i] *= q;
    }
    return OK;
}

// grating_energy_distr (rt_engine_func.h:75-78; rt_cuda_engine_surface.cu:
// 2098-2153,2190-2290): energy_distr[i] *= the blaze efficiency in `order`;
// angles in radians.
int oracle_grating_energy_distr(size_t n, const double* lambda, long order, double blaze_angle, double alpha,
                                double gamma, double gr_const, double rule_start, double rule_stop,
                                double* energy_distr) {
    const double rule_size = rule_stop - rule_start;
    for (size_t i = 0; i < n; ++i)
        energy_distr[i] *= grating_energy(lambda[i], order, blaze_angle, alpha, gamma, gr_const, rule_size);
    return OK;
}

// losses_comp's per-file computation (efficiency/losses_comp.cpp:60-90) on
// host arrays: lambda of all n rays (good first); ll[i] = i*nl-th of the
// sorted wavelengths, ratio[i] = count of ll[i] in the next nl sorted good
// wavelengths / nl.  The window is clipped to the good rays (the reference
// reads past their end when it runs over).
int oracle_loss_ratios(const double* lambda, uint64_t n, uint64_t n_good, uint64_t n_lambda, double* ll,
                       double* ratio) {
    if (n_lambda == 0 || n_good > n) return BAD_VALUE;
    std::vector<double> all(lambda, lambda + n), good(lambda, lambda + n_good);
    std::sort(all.begin(), all.end());
    std::sort(good.begin(), good.end());
    const size_t nl = n / n_lambda;
    for (size_t i = 0; i < n_lambda; ++i) ll[i] = all[i * nl];
    size_t cur = 0;
    for (size_t i = 0; i < n_lambda; ++i) {
        const size_t e = std::min(cur + nl, (size_t)n_good);
        const size_t cnt = (size_t)std::count(good.begin() + cur, good.begin() + e, ll[i]);
        ratio[i] = 1.0 * cnt / nl;
        cur += cnt;
        if (cur > n_good) break;
    }
    return OK;
}

// print_lambda's scan (tools/print_lambda.cpp:52-71): the distinct values of
// lambda[0, n_good) in order of first occurrence, the first one always, then
// stopping when their count equals n_lambda at the end of a step; at most
// cap values are written, *n_out is the count.
int oracle_unique_lambdas(const double* lambda, uint64_t n_good, uint64_t n_lambda, double* out, uint64_t cap,
                          uint64_t* n_out) {
    *n_out = 0;
    if (n_good == 0) return OK;
    std::vector<double> uniq{lambda[0]};
    for (size_t i = 1; i < n_good; ++i) {
        size_t j = 0;
        for (; j < uniq.size(); ++j)
            if (lambda[i] == uniq[j]) break;
        if (j == uniq.size()) uniq.push_back(lambda[i]);
        if (uniq.size() == n_lambda) break;
    }
    const size_t m = std::min((size_t)cap, uniq.size());
    std::copy(uniq.begin(), uniq.begin() + m, out);
    *n_out = m;
    return OK;
}

// Scheme::ComputeQE's curves (scheme.cpp:1249-1316) for explicit QE
// surfaces: per range, lambda_i = w1 + (w2-w1)/(N-1)*i and QE = 1, then per
// surface Surface::ApplyQE (surface.cpp:331-340: QE *= qe_curve(lambda)) and
// for a grating Grating::ApplyQE (surface.cpp:614-635: also *= its blaze
// efficiency in |order|, with SetRuleParams's conversions, surface.cpp:595-611).
// With more than one range, grating g takes its order from column 2 + g.
int oracle_qe_curves(const rtb_qe_surface* s, size_t n_s, const double* rows, size_t n_rows, size_t row_len,
                     size_t n_lambda, double* lambda, double* qe) {
    if (n_lambda < 2) return BAD_VALUE;
    for (size_t r = 0; r < n_rows; ++r) {
        const double* val = rows + r * row_len;
        double* lam = lambda + r * n_lambda;
        double* q = qe + r * n_lambda;
        double d_lambda = (val[1] - val[0]) / (n_lambda - 1);
        for (size_t i = 0; i < n_lambda; ++i) {
            lam[i] = val[0] + d_lambda * i;
            q[i] = 1.0;
        }
        size_t i_grating = 0;
        for (size_t k = 0; k < n_s; ++k) {
            int st = oracle_surface_QE(n_lambda, lam, q, &s[k].qe);
            if (st != OK) return st;
            if (s[k].type != RTB_GRATING) continue;
            long order = (long)s[k].order;
            if (n_rows > 1) order = static_cast<long>(val[i_grating + 2]);
            ++i_grating;
            double a = s[k].rule_start, b = s[k].rule_stop;
            a = a < 0.0 ? 0.0 : (a > 1.0 ? 1.0 : a);
            b = b < 0.0 ? 0.0 : (b > 1.0 ? 1.0 : b);
            if (a >= b) return BAD_VALUE;
            // `x*deg2rad` is x*RT_PI/180.0, evaluated left to right
            oracle_grating_energy_distr(n_lambda, lam, std::labs(order), s[k].blaze_deg * RTO_PI / 180.0,
                                        s[k].alpha_deg * RTO_PI / 180.0, s[k].gamma_deg * RTO_PI / 180.0,
                                        s[k].gr_const, a, b, q);
        }
    }
    return OK;
}

// ---- the trace ------------------------------------------------------------

// Per-ray formulation of Scheme::run over a batch of beams (host arrays,
// in place).  lost_counts (may be NULL) receives n_beams x (3*n_surfaces)
// counts of rays lost per stage.
int oracle_trace(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                 uint32_t fixes, int renorm_lost, const rtb_rays* rays, rtb_trace_stats* stats,
                 uint64_t* lost_counts) {
    std::vector<Prepared> S;
    int st = prepare(surfaces, n_surfaces, S);
    if (st != OK) return st;
    const std::vector<SurfConst> SC = surface_constants(S);
    const size_t n_stages = 3 * n_surfaces;
    std::vector<uint64_t> counts(n_beams * n_stages, 0);
    uint64_t ray_surfaces = 0, n_good = 0;
    std::atomic<int> err{0};
    for (size_t b = 0; b < n_beams; ++b) {
        const rtb_beam& bm = beams[b];
        if (bm.first_ray + bm.n_rays > rays->n) return BAD_VALUE;
        long orders[RTB_MAX_GRATINGS];
        for (int g = 0; g < RTB_MAX_GRATINGS; ++g) orders[g] = (long)bm.orders[g];
        std::vector<uint64_t> local(n_stages, 0);
        uint64_t rs = 0, ng = 0;
#pragma omp parallel
        {
            std::vector<uint64_t> mine(n_stages, 0);
            uint64_t my_rs = 0, my_ng = 0;
#pragma omp for schedule(static)
            for (long long ii = 0; ii < (long long)bm.n_rays; ++ii) {
                size_t i = bm.first_ray + (size_t)ii;
                Ray r{rays->X[i], rays->Y[i], rays->Z[i], rays->cX[i], rays->cY[i], rays->cZ[i]};
                int ls;
                int s2 = trace_ray(S, SC.data(), orders, bm.n_orders, rays->lambda[i], renorm_lost, fixes, r, ls,
                                   [](size_t) {});
                if (s2 != OK) { err = s2; continue; }
                rays->X[i] = r.X; rays->Y[i] = r.Y; rays->Z[i] = r.Z;
                rays->cX[i] = r.cX; rays->cY[i] = r.cY; rays->cZ[i] = r.cZ;
                rays->flag[i] = (ls == RTB_NOT_LOST) ? 1 : 0;
                if (rays->lost_stage) rays->lost_stage[i] = (uint8_t)ls;
                if (ls == RTB_NOT_LOST) { ++my_ng; my_rs += S.back().surfaces_upto; }
                else { ++mine[ls]; my_rs += S[ls / 3].surfaces_upto; }
            }
#pragma omp critical
            {
                for (size_t k = 0; k < n_stages; ++k) local[k] += mine[k];
                rs += my_rs;
                ng += my_ng;
            }
        }
        for (size_t k = 0; k < n_stages; ++k) counts[b * n_stages + k] = local[k];
        ray_surfaces += rs;
        n_good += ng;
    }
    if (err) return err;
    int failed_beam = -1, failed_stage = -1;
    for (size_t b = 0; b < n_beams && failed_beam < 0; ++b) {
        uint64_t alive = beams[b].n_rays;
        for (size_t k = 0; k < n_stages; ++k) {
            uint64_t lost = counts[b * n_stages + k];
            if (lost > 0 && lost == alive) { failed_beam = (int)b; failed_stage = (int)k; break; }
            alive -= lost;
        }
    }
    if (lost_counts) std::memcpy(lost_counts, counts.data(), counts.size() * sizeof(uint64_t));
    if (stats) {
        stats->ray_surfaces = ray_surfaces;
        stats->n_good = n_good;
        stats->failed_beam = failed_beam;
        stats->failed_stage = failed_stage;
    }
    if (failed_beam >= 0) return (failed_stage % 3 == 2) ? NO_GOOD_RAYS : NO_INTERSECTIONS;
    return OK;
}

// Algorithmic operation count of the reference's per-ray arithmetic
// (flop_count.hpp): every ray of `rays` (not modified) traced with the
// counting scalar, as oracle_trace traces it.  ops[k] (k < n_surfaces) sums
// the operations of surface k -- its transform, Normalize, intersection,
// aperture, action and Normalize -- over the rays that reach it, reached[k]
// counts those rays; ops[n_surfaces] holds the trailing Normalize calls of
// lost rays (renorm_lost).
int oracle_count_flops(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                       uint32_t fixes, int renorm_lost, const rtb_rays* rays, uint64_t* ops, uint64_t* reached) {
    std::vector<Prepared> S;
    int st = prepare(surfaces, n_surfaces, S);
    if (st != OK) return st;
    std::vector<SurfConstT<Flop>> SC(S.size());
    for (size_t k = 0; k < S.size(); ++k) SC[k] = SurfConstT<Flop>(S[k].sc);
    std::vector<uint64_t> tot_ops(n_surfaces + 1, 0), tot_reached(n_surfaces + 1, 0);
    std::atomic<int> err{0};
    for (size_t b = 0; b < n_beams; ++b) {
        const rtb_beam& bm = beams[b];
        if (bm.first_ray + bm.n_rays > rays->n) return BAD_VALUE;
        long orders[RTB_MAX_GRATINGS];
        for (int g = 0; g < RTB_MAX_GRATINGS; ++g) orders[g] = (long)bm.orders[g];
#pragma omp parallel
        {
            std::vector<uint64_t> my_ops(n_surfaces + 1, 0), my_reached(n_surfaces + 1, 0);
#pragma omp for schedule(static)
            for (long long ii = 0; ii < (long long)bm.n_rays; ++ii) {
                const size_t i = bm.first_ray + (size_t)ii;
                if (rays->flag && rays->flag[i] != 1) continue;
                RayT<Flop> r{rays->X[i], rays->Y[i], rays->Z[i], rays->cX[i], rays->cY[i], rays->cZ[i]};
                int ls;
                size_t cur = 0;
                uint64_t mark = Flop::n;
                auto at = [&](size_t k) {
                    if (k > 0) my_ops[cur] += Flop::n - mark;
                    mark = Flop::n;
                    cur = k;
                    ++my_reached[k];
                };
                int s2 = trace_ray(S, SC.data(), orders, bm.n_orders, Flop(rays->lambda[i]), renorm_lost, fixes, r,
                                   ls, at);
                my_ops[cur] += Flop::n - mark;
                if (s2 != OK) err = s2;
            }
#pragma omp critical
            for (size_t k = 0; k <= n_surfaces; ++k) {
                tot_ops[k] += my_ops[k];
                tot_reached[k] += my_reached[k];
            }
        }
    }
    if (err) return err;
    for (size_t k = 0; k <= n_surfaces; ++k) {
        if (ops) ops[k] = tot_ops[k];
        if (reached) reached[k] = tot_reached[k];
    }
    return OK;
}

// Statement-for-statement replica of the per-surface loop for ONE beam
// (scheme.cpp:983-1055 with beam.cpp:527-598,601-633, surface.cpp:244-321,
// 385-396,453-472,563-585).  Arrays hold n rays, all good on entry; on exit
// they are in the reference's order and *n_good_out is N_good_rays.
int oracle_trace_literal(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beam,
                         uint32_t fixes, double* X, double* Y, double* Z, double* cX, double* cY,
                         double* cZ, double* lambda, char* flag, size_t n, size_t* n_good_out) {
    std::vector<Prepared> S;
    int st = prepare(surfaces, n_surfaces, S);
    if (st != OK) return st;
    double* arr[7] = {X, Y, Z, cX, cY, cZ, lambda};
    auto swapper = [&](size_t a, size_t b) { for (double* v : arr) std::swap(v[a], v[b]); };
    size_t ng = n;
    for (size_t i = 0; i < n; ++i) flag[i] = 1;
    long orders[RTB_MAX_GRATINGS];
    for (int g = 0; g < RTB_MAX_GRATINGS; ++g) orders[g] = (long)beam->orders[g];
    for (size_t k = 0; k < S.size(); ++k) {
        const Prepared& p = S[k];
        for (size_t i = 0; i < ng; ++i) {            // Beam::Transform: good prefix
            Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
            transform(p.tc, r);
            X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z; cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
        }
        for (size_t i = 0; i < n; ++i) normalize(cX[i], cY[i], cZ[i]);   // all rays
        if (!p.non_aux) continue;
        // Intersection
        size_t bad = 0;
        for (size_t i = 0; i < ng; ++i) {
            Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
            if (!intersect(p.kind, p.sc, fixes, r)) { flag[i] = 0; ++bad; }
            X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z;
        }
        if (bad) {
            if (bad == ng) { *n_good_out = ng; return NO_INTERSECTIONS; }
            ng = rearrange(flag, ng, swapper);
        }
        // Aperture
        bad = 0;
        for (size_t i = 0; i < ng; ++i)
            if (!aperture_pass(p.type == Shade, p.shape, p.size, p.center, X[i], Y[i])) { flag[i] = 0; ++bad; }
        if (bad) {
            if (bad == ng) { *n_good_out = ng; return NO_INTERSECTIONS; }
            ng = rearrange(flag, ng, swapper);
        }
        // Action
        bad = 0;
        for (size_t i = 0; i < ng; ++i) {
            Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
            int a = action(p, p.sc, orders, beam->n_orders, lambda[i], r);
            if (a == NO_GOOD_RAYS) { flag[i] = 0; ++bad; }
            else if (a != OK) { *n_good_out = ng; return a; }
            cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
        }
        if (bad) {
            if (bad == ng) { *n_good_out = ng; return NO_GOOD_RAYS; }
            ng = rearrange(flag, ng, swapper);
        }
        for (size_t i = 0; i < n; ++i) normalize(cX[i], cY[i], cZ[i]);
    }
    *n_good_out = ng;
    return OK;
}

// Order replay: from per-ray lost stages (ray index order), the positions the
// reference's successive Rearrange calls give the rays of one beam.
// order[k] = ray index (0-based within the beam) at position k.
int oracle_reference_order(size_t n, size_t n_stages, const uint8_t* lost_stage, uint32_t* order,
                           size_t* n_good_out) {
    for (size_t i = 0; i < n; ++i) order[i] = (uint32_t)i;
    std::vector<char> fl(n);
    size_t ng = n;
    for (size_t s = 0; s < n_stages; ++s) {
        size_t bad = 0;
        for (size_t k = 0; k < ng; ++k) {
            bool lost = lost_stage[order[k]] == s;
            fl[k] = lost ? 0 : 1;
            bad += lost;
        }
        if (!bad) continue;
        ng = rearrange(fl.data(), ng, [&](size_t a, size_t b) { std::swap(order[a], order[b]); });
    }
    *n_good_out = ng;
    return OK;
}

// Apply the reference's remaining Normalize calls to lost rays, as
// oracle_trace does with renorm_lost; exposed for tests.
int oracle_renormalize_count(const rtb_surface* surfaces, size_t n_surfaces, int stage) {
    std::vector<Prepared> S;
    if (prepare(surfaces, n_surfaces, S) != OK) return -1;
    return S[stage / 3].renorm_after;
}

// Frame counts of good rays on the CCD (uint32, no reference counterpart).
int oracle_ccd_frame(const rtb_rays* rays, const rtb_ccd* ccd, uint32_t* counts, uint64_t* n_outside) {
    uint64_t outside = 0;
    for (size_t i = 0; i < rays->n; ++i) {
        if (rays->flag[i] != 1) continue;
        uint32_t ix, iy;
        ccd_coords(rays->X[i], rays->Y[i], ccd->xsize, ccd->ysize, ccd->xpix, ccd->ypix, ix, iy);
        if (ix >= ccd->xdim || iy >= ccd->ydim) { ++outside; continue; }
        counts[(size_t)iy * ccd->xdim + ix] += 1;
    }
    if (n_outside) *n_outside += outside;
    return OK;
}

}  // extern "C"
