// rt_engine_b200.cpp -- the reference's engine API on the B200 engine.
//
// Implements every prototype of common-lib/rt_engine_func.h:25-104 with the
// reference's own C++ signatures by calling the C ABI of librtb200.so
// (include/rtb.h).  A build of amirych/rt compiles this file (with its
// common-lib headers on the include path) and links librtb200.so in place of
// the objects of cuda_engine/, leaving Beam, Surface, TabulatedFunction,
// Scheme, ray-tracing and ccd_frame unchanged.
//
// TabulatedFunction keeps its knots private (tabulated_function.h:47-49).
// The engine evaluates n(lambda), QE(lambda) and spectra on the device from
// the knots, so this file reads them through member pointers obtained by
// explicit template instantiation, which the language exempts from access
// checking ([temp.explicit]); tabulated_function.h is not edited.
#include "rt_engine_func.h"
#include "tabulated_function.h"
#include "rtb.h"

#include <chrono>
#include <sstream>
#include <string>
#include <vector>

namespace {

template <typename Tag, typename Tag::type M>
struct PrivateMember {
    friend typename Tag::type member_ptr(Tag) { return M; }
};

struct TF_single {
    typedef bool TabulatedFunction::*type;
    friend type member_ptr(TF_single);
};
struct TF_x {
    typedef std::vector<real_t> TabulatedFunction::*type;
    friend type member_ptr(TF_x);
};
struct TF_y {
    typedef std::vector<real_t> TabulatedFunction::*type;
    friend type member_ptr(TF_y);
};
struct TF_y2 {
    typedef std::vector<real_t> TabulatedFunction::*type;
    friend type member_ptr(TF_y2);
};
template struct PrivateMember<TF_single, &TabulatedFunction::SingleValue>;
template struct PrivateMember<TF_x, &TabulatedFunction::x>;
template struct PrivateMember<TF_y, &TabulatedFunction::y>;
template struct PrivateMember<TF_y2, &TabulatedFunction::dy2>;

// rtb_table view of a TabulatedFunction: a single value is n == 1.
rtb_table table_of(TabulatedFunction& f) {
    const std::vector<real_t>& x = f.*member_ptr(TF_x());
    const std::vector<real_t>& y = f.*member_ptr(TF_y());
    const std::vector<real_t>& y2 = f.*member_ptr(TF_y2());
    rtb_table t;
    t.n = (f.*member_ptr(TF_single())) ? (y.empty() ? 0 : 1) : y.size();
    t.x = x.data();
    t.y = y.data();
    t.y2 = y2.data();
    return t;
}

// Status -> RT_engine_error.  A wavelength outside a table makes the
// reference throw TabulatedFunction::bad_tab_func(OutOfRange) from inside
// the engine call (tabulated_function.cpp:179-181); the shim does the same.
RT_engine_error to_engine_error(int st) {
    switch (st) {
        case RTB_OK: return ENGINE_ERROR_OK;
        case RTB_INIT_FAILED: return ENGINE_ERROR_INIT_FAILED;
        case RTB_BAD_ALLOC: return ENGINE_ERROR_BAD_ALLOC;
        case RTB_BAD_VALUE: return ENGINE_ERROR_BAD_VALUE;
        case RTB_OUT_OF_RANGE: throw TabulatedFunction::bad_tab_func(TabulatedFunction::OutOfRange);
        default: return ENGINE_ERROR_FAILED;
    }
}

// The reference seeds its generators with the clock (rt_cuda_engine_beam.cu:270-275).
uint64_t clock_seed() {
    return (uint64_t)std::chrono::steady_clock::now().time_since_epoch().count();
}

}  // namespace

RT_engine_error rt_engine_init() { return to_engine_error(rtb_init()); }

RT_engine_error rt_engine_info(list<string>& info_str) {
    char buf[1024];
    int st = rtb_info(buf, sizeof(buf));
    if (st != RTB_OK) return to_engine_error(st);
    info_str.clear();
    std::istringstream in(buf);
    std::string line;
    while (std::getline(in, line))
        if (!line.empty()) info_str.push_back(line);
    return ENGINE_ERROR_OK;
}

RT_engine_error beam_random(Beam::BeamShape shape, real_t* params, real_t* center, size_t Nrays, real_t* X, real_t* Y,
                            real_t* Z) {
    return to_engine_error(rtb_beam_random((int)shape, params, center, Nrays, X, Y, Z, clock_seed(), 0));
}

RT_engine_error beam_conic_cosins(size_t Nrays, real_t conic_angle, real_t* X, real_t* Y, real_t* cX, real_t* cY,
                                  real_t* cZ) {
    return to_engine_error(rtb_beam_conic_cosins(Nrays, conic_angle, X, Y, cX, cY, cZ));
}

RT_engine_error beam_gauss_cosins(size_t Nrays, real_t fwhm, real_t* cX, real_t* cY, real_t* cZ) {
    return to_engine_error(rtb_beam_gauss_cosins(Nrays, fwhm, cX, cY, cZ, clock_seed()));
}

RT_engine_error uniform_range_beam(size_t Nrays, real_t* range, real_t* lambda) {
    return to_engine_error(rtb_uniform_range_beam(Nrays, range, lambda));
}

RT_engine_error random_range_beam(size_t Nrays, real_t* range, real_t* lambda) {
    return to_engine_error(rtb_random_range_beam(Nrays, range, lambda, clock_seed()));
}

RT_engine_error beam_transform(size_t Nrays, real_t* angles, real_t* dist, real_t* X, real_t* Y, real_t* Z, real_t* cX,
                               real_t* cY, real_t* cZ) {
    return to_engine_error(rtb_beam_transform(Nrays, angles, dist, X, Y, Z, cX, cY, cZ));
}

RT_engine_error surface_intersection(Surface::SurfaceClass surf_class, real_t* params, size_t Nrays, real_t* X,
                                     real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ, size_t* N_bad,
                                     beam_flag_t* flag) {
    return to_engine_error(rtb_surface_intersection((int)surf_class, params, Nrays, X, Y, Z, cX, cY, cZ, N_bad, flag));
}

RT_engine_error surface_reflection(Surface::SurfaceClass surf_class, real_t* params, size_t Nrays, real_t* X,
                                   real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ) {
    return to_engine_error(rtb_surface_reflection((int)surf_class, params, Nrays, X, Y, Z, cX, cY, cZ));
}

RT_engine_error surface_refraction(Surface::SurfaceClass surf_class, real_t* params, size_t Nrays, real_t* X,
                                   real_t* Y, real_t* Z, real_t* cX, real_t* cY, real_t* cZ, real_t* lambda,
                                   TabulatedFunction& n1, TabulatedFunction& n2, size_t* N_bad, beam_flag_t* flag) {
    rtb_table t1 = table_of(n1), t2 = table_of(n2);
    return to_engine_error(
        rtb_surface_refraction((int)surf_class, params, Nrays, X, Y, Z, cX, cY, cZ, lambda, &t1, &t2, N_bad, flag));
}

RT_engine_error surface_diffration(Surface::SurfaceClass surf_class, Grating::GratingType gr_type, real_t* params,
                                   long diff_order, real_t gr_constant, size_t Nrays, real_t* X, real_t* Y, real_t* Z,
                                   real_t* cX, real_t* cY, real_t* cZ, real_t* lambda, TabulatedFunction& n1,
                                   TabulatedFunction& n2, size_t* N_bad, beam_flag_t* flag) {
    rtb_table t1 = table_of(n1), t2 = table_of(n2);
    return to_engine_error(rtb_surface_diffration((int)surf_class, (int)gr_type, params, diff_order, gr_constant, Nrays,
                                                  X, Y, Z, cX, cY, cZ, lambda, &t1, &t2, N_bad, flag));
}

RT_engine_error surface_QE(size_t N, real_t* lambda, real_t* spec, TabulatedFunction& QE) {
    rtb_table t = table_of(QE);
    return to_engine_error(rtb_surface_QE(N, lambda, spec, &t));
}

RT_engine_error grating_energy_distr(size_t N, real_t* lambda, long order, real_t blaze_angle, real_t alpha,
                                     real_t gamma, real_t gr_const, real_t rule_start, real_t rule_stop,
                                     real_t* energy_distr) {
    return to_engine_error(rtb_grating_energy_distr(N, lambda, order, blaze_angle, alpha, gamma, gr_const, rule_start,
                                                    rule_stop, energy_distr));
}

void rt_engine_free_vector(real_t* data) { rtb_free_vector(data); }

real_t* rt_engine_alocate_vector(size_t N_elem) { return rtb_alocate_vector(N_elem); }

RT_engine_error spline_init(size_t N, real_t* x, real_t* y, real_t* y2) {
    return to_engine_error(rtb_spline_init(N, x, y, y2));
}

RT_engine_error ccd_coordinates(size_t Nrays, real_t* X, real_t* Y, real_t ccd_xsize, real_t ccd_ysize,
                                real_t ccd_xpix, real_t ccd_ypix, unsigned int* ccd_X, unsigned int* ccd_Y) {
    return to_engine_error(rtb_ccd_coordinates(Nrays, X, Y, ccd_xsize, ccd_ysize, ccd_xpix, ccd_ypix, ccd_X, ccd_Y));
}

RT_engine_error compute_ccd_image(size_t Nrays, unsigned int* ccd_X, unsigned int* ccd_Y, real_t* lambda,
                                  TabulatedFunction& QE, TabulatedFunction& incident_spec, size_t ccd_xdim,
                                  size_t ccd_ydim, real_t ccd_xpix, real_t ccd_ypix, real_t* image) {
    rtb_table q = table_of(QE), s = table_of(incident_spec);
    return to_engine_error(rtb_compute_ccd_image(Nrays, ccd_X, ccd_Y, lambda, &q, &s, ccd_xdim, ccd_ydim, ccd_xpix,
                                                 ccd_ypix, image, nullptr));
}
