// oracle_engine.cpp -- the CPU oracle behind the reference's engine API.
//
// TEST INFRASTRUCTURE ONLY.  Implements the prototypes of
// common-lib/rt_engine_func.h:25-104 with the oracle's restated arithmetic
// (rt_oracle.hpp), so that the reference's own host classes (Beam, Surface,
// TabulatedFunction, compiled from the reference sources by oracle/Makefile)
// can run the per-surface loop on the CPU.  Comparing that run with
// oracle_trace_literal pins the oracle's restatement of the host loops
// (Normalize, Rearrange, ApplyConstrains, the transform plumbing) to the
// reference's own code.  Built only into oracle/_ref/.
#include "rt_engine_func.h"
#include "rt_oracle.hpp"

#include <cstdlib>
#include <vector>

using namespace rto;

RT_engine_error rt_engine_init() { return ENGINE_ERROR_OK; }

RT_engine_error rt_engine_info(list<string>& info_str) {
    info_str.clear();
    info_str.push_back("CPU oracle engine (test infrastructure)");
    return ENGINE_ERROR_OK;
}

RT_engine_error beam_random(Beam::BeamShape shape, real_t* params, real_t* center, size_t Nrays,
                            real_t* X, real_t* Y, real_t* Z) {
    if (shape != Beam::Circle) return ENGINE_ERROR_BAD_VALUE;
    for (size_t i = 0; i < Nrays; ++i) {
        double u1, u2;
        ray_uniforms(0x5eed, 0, i, u1, u2);
        disk_position(params, center, u1, u2, X[i], Y[i], Z[i]);
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error beam_conic_cosins(size_t, real_t, real_t*, real_t*, real_t*, real_t*, real_t*) {
    return ENGINE_ERROR_FAILED;
}

RT_engine_error beam_gauss_cosins(size_t, real_t, real_t*, real_t*, real_t*) { return ENGINE_ERROR_FAILED; }

RT_engine_error uniform_range_beam(size_t Nrays, real_t* range, real_t* lambda) {
    for (size_t j = 0; j < Nrays; ++j) lambda[j] = uniform_lambda(range, Nrays, j);
    return ENGINE_ERROR_OK;
}

RT_engine_error random_range_beam(size_t Nrays, real_t* range, real_t* lambda) {
    for (size_t i = 0; i < Nrays; ++i) {
        double u1, u2;
        ray_uniforms(0x5eed, 1, i, u1, u2);
        lambda[i] = (range[1] - range[0]) * u1 + range[0];
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error beam_transform(size_t Nrays, real_t* angles, real_t* dist, real_t* X, real_t* Y, real_t* Z,
                               real_t* cX, real_t* cY, real_t* cZ) {
    TransformConst t = make_transform(angles, dist);
    for (size_t i = 0; i < Nrays; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        transform(t, r);
        X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z; cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error surface_intersection(Surface::SurfaceClass surf_class, real_t* params, size_t Nrays,
                                     real_t* X, real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ,
                                     size_t* N_bad, beam_flag_t* flag) {
    if (surf_class == Surface::AuxClass) return ENGINE_ERROR_OK;
    SurfConst s;
    if (make_surf_const(surf_class, params, s) != OK) return ENGINE_ERROR_BAD_VALUE;
    IsectKind kind = intersection_kind(surf_class, params);
    for (size_t i = 0; i < Nrays; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        if (!intersect(kind, s, 0, r)) { flag[i] = 0; ++*N_bad; }
        X[i] = r.X; Y[i] = r.Y; Z[i] = r.Z;
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error surface_reflection(Surface::SurfaceClass surf_class, real_t* params, size_t Nrays,
                                   real_t* X, real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ) {
    SurfConst s;
    if (make_surf_const(surf_class, params, s) != OK) return ENGINE_ERROR_BAD_VALUE;
    for (size_t i = 0; i < Nrays; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        reflect(surf_class, s, r);
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    return ENGINE_ERROR_OK;
}

// Refraction and diffraction evaluate n(lambda) through the reference's own
// TabulatedFunction::operator[], per ray, as the reference engine does
// (surface.cu:1094-1097,1565-1569,1608-1610).
RT_engine_error surface_refraction(Surface::SurfaceClass surf_class, real_t* params, size_t Nrays,
                                   real_t* X, real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ,
                                   real_t* lambda, TabulatedFunction& n1, TabulatedFunction& n2,
                                   size_t* N_bad, beam_flag_t* flag) {
    SurfConst s;
    if (make_surf_const(surf_class, params, s) != OK) return ENGINE_ERROR_BAD_VALUE;
    std::vector<double> mu(Nrays);
    for (size_t i = 0; i < Nrays; ++i) {
        mu[i] = n1[lambda[i]];
        mu[i] /= n2[lambda[i]];
    }
    for (size_t i = 0; i < Nrays; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        if (!refract(surf_class, s, mu[i], r)) { flag[i] = 0; ++*N_bad; }
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error surface_diffration(Surface::SurfaceClass surf_class, Grating::GratingType gr_type,
                                   real_t* params, long diff_order, real_t gr_constant, size_t Nrays,
                                   real_t* X, real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ,
                                   real_t* lambda, TabulatedFunction& n1, TabulatedFunction& n2,
                                   size_t* N_bad, beam_flag_t* flag) {
    SurfConst s;
    if (make_surf_const(surf_class, params, s) != OK) return ENGINE_ERROR_BAD_VALUE;
    std::vector<double> mu(Nrays, 0.0), L(Nrays);
    for (size_t i = 0; i < Nrays; ++i) {
        if (gr_type == Grating::Transparent) {
            mu[i] = n1[lambda[i]];
            mu[i] /= n2[lambda[i]];
        }
        L[i] = diff_order * lambda[i] / n2[lambda[i]] / gr_constant;
    }
    for (size_t i = 0; i < Nrays; ++i) {
        Ray r{X[i], Y[i], Z[i], cX[i], cY[i], cZ[i]};
        if (!diffract(surf_class, gr_type, s, mu[i], L[i], r)) { flag[i] = 0; ++*N_bad; }
        cX[i] = r.cX; cY[i] = r.cY; cZ[i] = r.cZ;
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error surface_QE(size_t N, real_t* lambda, real_t* spec, TabulatedFunction& QE) {
    for (size_t i = 0; i < N; ++i) spec[i] *= QE[lambda[i]];
    return ENGINE_ERROR_OK;
}

RT_engine_error grating_energy_distr(size_t N, real_t* lambda, long order, real_t blaze_angle, real_t alpha,
                                     real_t gamma, real_t gr_const, real_t rule_start, real_t rule_stop,
                                     real_t* energy_distr) {
    const real_t rule_size = rule_stop - rule_start;
    for (size_t i = 0; i < N; ++i)
        energy_distr[i] *= rto::grating_energy(lambda[i], order, blaze_angle, alpha, gamma, gr_const, rule_size);
    return ENGINE_ERROR_OK;
}

void rt_engine_free_vector(real_t* data) { free(data); }

real_t* rt_engine_alocate_vector(size_t N_elem) { return (real_t*)malloc(sizeof(real_t) * N_elem); }

RT_engine_error spline_init(size_t N, real_t* x, real_t* y, real_t* y2) {
    if (N < 4) return ENGINE_ERROR_BAD_VALUE;
    rto::spline_init(N, x, y, y2);
    return ENGINE_ERROR_OK;
}

RT_engine_error ccd_coordinates(size_t Nrays, real_t* X, real_t* Y, real_t ccd_xsize, real_t ccd_ysize,
                                real_t ccd_xpix, real_t ccd_ypix, unsigned int* ccd_X, unsigned int* ccd_Y) {
    for (size_t i = 0; i < Nrays; ++i) {
        uint32_t a, b;
        ccd_coords(X[i], Y[i], ccd_xsize, ccd_ysize, ccd_xpix, ccd_ypix, a, b);
        ccd_X[i] = a; ccd_Y[i] = b;
    }
    return ENGINE_ERROR_OK;
}

RT_engine_error compute_ccd_image(size_t Nrays, unsigned int* ccd_X, unsigned int* ccd_Y, real_t* lambda,
                                  TabulatedFunction& QE, TabulatedFunction& incident_spec, size_t ccd_xdim,
                                  size_t ccd_ydim, real_t ccd_xpix, real_t ccd_ypix, real_t* image) {
    double pix_area = ccd_xpix * ccd_ypix * 1.0E-2;
    for (size_t i = 0; i < Nrays; ++i) {
        double q = QE[lambda[i]];
        double sp = incident_spec[lambda[i]] * lambda[i];
        if (ccd_X[i] >= ccd_xdim || ccd_Y[i] >= ccd_ydim) continue;
        unsigned int index = ccd_Y[i] * (unsigned int)ccd_xdim + ccd_X[i];
        image[index] += sp / HC * q * pix_area;
    }
    return ENGINE_ERROR_OK;
}
