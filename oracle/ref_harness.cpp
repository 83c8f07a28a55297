// ref_harness.cpp -- drives the reference's own host classes.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
// reference's common-lib sources (beam.cpp, surface.cpp,
// tabulated_function.cpp, ascii_file.cpp) and one engine behind
// common-lib/rt_engine_func.h:
//   harness_cpu    -- the CPU oracle (oracle_engine.cpp); runs anywhere;
//   harness_refgpu -- the reference cuda_engine built for sm_100a (GPU only);
//   harness_b200   -- the B200 engine through rt_b200/shim (GPU only).
// It replays the per-surface loop of Scheme::run (scheme.cpp:983-1055)
// through the public Beam/Surface API on an injected beam (the reference's
// beam generator is clock-seeded, beam.cu:270-275), and writes the result
// with Beam::Save (beam.cpp:636-715).  Scheme XML parsing (Mini-XML) is not
// involved: surfaces are built with their constructors.
//
// Usage:
//   harness trace <spec.txt> <beam.bin> <out.dat>
//   harness tabfunc <table.txt> <xs.bin> <out.bin>
//   harness ccd <xy.bin> <xsize> <ysize> <xpix> <ypix> <out.bin>
//   harness qe <qe_spec.txt> <out.bin>
// Exit codes: 0 ok, 5 NoIntersections, 6 NoGoodRays, 7 table out of range,
// 4 BadRuleParams, 3 other engine failure, 2 usage / IO.
#include "beam.h"
#include "surface.h"
#include "tabulated_function.h"
#include "rt_engine_func.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

// Read access to Beam's private arrays without editing beam.h: an explicit
// instantiation may name private members ([temp.explicit]), and the friend
// function it defines hands out the member pointer.
template <typename Tag, typename Tag::type M>
struct PrivateMember {
    friend typename Tag::type member_ptr(Tag) { return M; }
};
#define RTB_PRIVATE(NAME, CLASS, TYPE, MEMBER)                 \
    struct NAME {                                              \
        typedef TYPE CLASS::*type;                             \
        friend type member_ptr(NAME);                          \
    };                                                         \
    template struct PrivateMember<NAME, &CLASS::MEMBER>;

RTB_PRIVATE(B_Nrays, Beam, size_t, Nrays)
RTB_PRIVATE(B_Ngood, Beam, size_t, N_good_rays)
RTB_PRIVATE(B_Nlambda, Beam, size_t, N_lambda)
RTB_PRIVATE(B_X, Beam, real_t*, X)
RTB_PRIVATE(B_Y, Beam, real_t*, Y)
RTB_PRIVATE(B_Z, Beam, real_t*, Z)
RTB_PRIVATE(B_cX, Beam, real_t*, cX)
RTB_PRIVATE(B_cY, Beam, real_t*, cY)
RTB_PRIVATE(B_cZ, Beam, real_t*, cZ)
RTB_PRIVATE(B_lambda, Beam, real_t*, lambda)
RTB_PRIVATE(B_flag, Beam, beam_flag_t*, flag)

static int usage() {
    std::fprintf(stderr, "usage: harness trace|tabfunc|ccd ...\n");
    return 2;
}

static bool read_doubles(FILE* f, double* p, size_t n) { return std::fread(p, sizeof(double), n, f) == n; }

struct IndexSpec {
    bool is_file = false;
    double value = 1.0;
    std::string file;
};

static IndexSpec parse_index(const std::string& tok) {
    IndexSpec s;
    if (tok.compare(0, 2, "f:") == 0) { s.is_file = true; s.file = tok.substr(2); }
    else s.value = std::atof(tok.substr(2).c_str());
    return s;
}

static Surface* make_surface(std::istream& in, std::vector<long>& grating_orders_unused) {
    (void)grating_orders_unused;
    int cls, type, shape, gtype;
    long order;
    double gr_const;
    size_t np;
    in >> cls >> type >> shape >> gtype >> order >> gr_const >> np;
    std::vector<real_t> params(np);
    for (size_t i = 0; i < np; ++i) in >> params[i];
    std::vector<real_t> size(2), center(2), dist(3), ang(3);
    in >> size[0] >> size[1] >> center[0] >> center[1] >> dist[0] >> dist[1] >> dist[2] >> ang[0] >> ang[1] >> ang[2];
    std::string t1, t2;
    in >> t1 >> t2;
    if (!in) return nullptr;
    IndexSpec n1 = parse_index(t1), n2 = parse_index(t2);
    Surface::SurfaceClass cl = (Surface::SurfaceClass)cls;
    Surface::SurfaceShape sh = (Surface::SurfaceShape)shape;
    Surface* s = nullptr;
    switch ((Surface::SurfaceType)type) {
        case Surface::Mirror: s = new Mirror(cl, sh); break;
        case Surface::Lens:
            if (!n1.is_file && !n2.is_file) s = new Lens(cl, sh, n1.value, n2.value);
            else if (!n1.is_file) s = new Lens(cl, sh, n1.value, n2.file.c_str());
            else if (!n2.is_file) s = new Lens(cl, sh, n1.file.c_str(), n2.value);
            else s = new Lens(cl, sh, n1.file.c_str(), n2.file.c_str());
            break;
        case Surface::Grating: {
            std::vector<long> ord(1, order);
            Grating::GratingType gt = (Grating::GratingType)gtype;
            if (!n1.is_file && !n2.is_file) s = new Grating(cl, sh, gt, ord, gr_const, n1.value, n2.value);
            else if (!n1.is_file) s = new Grating(cl, sh, gt, ord, gr_const, n1.value, n2.file.c_str());
            else if (!n2.is_file) s = new Grating(cl, sh, gt, ord, gr_const, n1.file.c_str(), n2.value);
            else s = new Grating(cl, sh, gt, ord, gr_const, n1.file.c_str(), n2.file.c_str());
            break;
        }
        case Surface::Stop: s = new Stop(cl, sh); break;
        case Surface::Shade: s = new Shade(cl, sh); break;
        case Surface::Detector: s = new Surface(cl, Surface::Detector, sh); break;
        case Surface::AuxType: s = new Aux(); break;
        default: return nullptr;
    }
    s->SetDistance(dist);
    s->SetAngles(ang);
    if (s->GetType() != Surface::AuxType) {
        s->SetParams(params);
        s->SetGeometry(size, center);
    }
    return s;
}

static int run_trace(const char* spec_path, const char* beam_path, const char* out_path) {
    std::ifstream spec(spec_path);
    if (!spec) return 2;
    size_t nsurf;
    spec >> nsurf;
    std::vector<Surface*> scheme;
    std::vector<long> unused;
    for (size_t k = 0; k < nsurf; ++k) {
        Surface* s = make_surface(spec, unused);
        if (!s) return 2;
        scheme.push_back(s);
    }
    size_t n_orders = 0;
    spec >> n_orders;
    std::vector<long> orders(n_orders);
    for (size_t i = 0; i < n_orders; ++i) spec >> orders[i];

    FILE* f = std::fopen(beam_path, "rb");
    if (!f) return 2;
    uint64_t n;
    if (std::fread(&n, sizeof(n), 1, f) != 1) return 2;
    Beam beam(Beam::Parallel, Beam::Circle, Beam::Random, Beam::UniformDistr);
    beam.*member_ptr(B_Nrays()) = n;
    beam.*member_ptr(B_Ngood()) = n;
    beam.*member_ptr(B_Nlambda()) = 1;
    real_t** arrays[7] = {&(beam.*member_ptr(B_X())), &(beam.*member_ptr(B_Y())), &(beam.*member_ptr(B_Z())),
                          &(beam.*member_ptr(B_cX())), &(beam.*member_ptr(B_cY())), &(beam.*member_ptr(B_cZ())),
                          &(beam.*member_ptr(B_lambda()))};
    for (real_t** a : arrays) {
        *a = rt_engine_alocate_vector(n);
        if (!*a || !read_doubles(f, *a, n)) return 2;
    }
    std::fclose(f);
    beam_flag_t*& flag = beam.*member_ptr(B_flag());
    flag = new beam_flag_t[n];
    for (size_t i = 0; i < n; ++i) flag[i] = 1;

    int rc = 0;
    const auto t0 = std::chrono::steady_clock::now();
    try {
        size_t i_grating = 0;
        for (Surface* s : scheme) {       // scheme.cpp:983-1055
            beam.Transform(*s);
            beam.Normalize();
            if (s->GetType() != Surface::AuxType) {
                s->Intersection(beam);
                s->ApplyConstrains(beam);
                if (s->GetType() == Surface::Grating && n_orders > 0) {
                    static_cast<Grating*>(s)->SetOrder(orders[i_grating]);
                    ++i_grating;
                }
                s->Action(beam);
                beam.Normalize();
            }
        }
        // wall time of the surface loop: the engine calls with their host
        // copies and the host loops of Beam and Surface, as Scheme::run runs them
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "trace_seconds=%.6f good=%zu\n", sec, (size_t)beam.GetNumberOfGoodRays());
        beam.Save(out_path);
    } catch (Surface::bad_surface& e) {
        Surface::SurfaceError err = e.surface_error();
        rc = (err == Surface::NoIntersections) ? 5 : (err == Surface::NoGoodRays) ? 6 : 3;
    } catch (TabulatedFunction::bad_tab_func& e) {
        rc = (e.bad_tab_func_error() == TabulatedFunction::OutOfRange) ? 7 : 3;
    } catch (...) {
        rc = 3;
    }
    for (Surface* s : scheme) delete s;
    return rc;
}

static int run_tabfunc(const char* table_path, const char* xs_path, const char* out_path) {
    FILE* f = std::fopen(xs_path, "rb");
    if (!f) return 2;
    uint64_t n;
    if (std::fread(&n, sizeof(n), 1, f) != 1) return 2;
    std::vector<double> xs(n), ys(n), ok(n);
    if (!read_doubles(f, xs.data(), n)) return 2;
    std::fclose(f);
    try {
        TabulatedFunction tf(table_path);
        for (size_t i = 0; i < n; ++i) {
            try { ys[i] = tf[xs[i]]; ok[i] = 1.0; }
            catch (TabulatedFunction::bad_tab_func&) { ys[i] = 0.0; ok[i] = 0.0; }
        }
    } catch (...) {
        return 3;
    }
    FILE* o = std::fopen(out_path, "wb");
    if (!o) return 2;
    std::fwrite(ys.data(), sizeof(double), n, o);
    std::fwrite(ok.data(), sizeof(double), n, o);
    std::fclose(o);
    return 0;
}

static int run_ccd(int argc, char** argv) {
    if (argc < 8) return usage();
    FILE* f = std::fopen(argv[2], "rb");
    if (!f) return 2;
    uint64_t n;
    if (std::fread(&n, sizeof(n), 1, f) != 1) return 2;
    std::vector<double> X(n), Y(n);
    if (!read_doubles(f, X.data(), n) || !read_doubles(f, Y.data(), n)) return 2;
    std::fclose(f);
    std::vector<unsigned int> ix(n), iy(n);
    RT_engine_error e = ccd_coordinates(n, X.data(), Y.data(), std::atof(argv[3]), std::atof(argv[4]),
                                        std::atof(argv[5]), std::atof(argv[6]), ix.data(), iy.data());
    if (e != ENGINE_ERROR_OK) return 3;
    FILE* o = std::fopen(argv[7], "wb");
    if (!o) return 2;
    std::fwrite(ix.data(), sizeof(unsigned int), n, o);
    std::fwrite(iy.data(), sizeof(unsigned int), n, o);
    std::fclose(o);
    return 0;
}

// Scheme::ComputeQE after its XML pass (scheme.cpp:1164-1201 for the
// surfaces, 1249-1334 for the curves and the QE file), on surfaces read from
// a text spec:
//   n_lambda n_rows row_len   then n_rows rows of row_len numbers
//   n_surfaces                then per surface:
//   type qe_token             (type 0 MIRROR, 1 LENS, 2 GRATING, 5 DETECTOR;
//                              qe_token v:<number> or f:<table file>)
//   and for a grating:  order const alpha gamma blaze_angle n_rule rule_1 .. rule_n
// The surfaces are built as ComputeQE builds them: a grating as
// Grating(Plane, Rectangle, Reflective, {order}, const, 1, 1) with
// SetRuleParams, every other type as Surface(Plane, Mirror, Circle).
static int run_qe(const char* spec_path, const char* out_path) {
    std::ifstream spec(spec_path);
    if (!spec) return 2;
    size_t n_lambda, n_rows, row_len, n_s;
    spec >> n_lambda >> n_rows >> row_len;
    std::vector<std::vector<real_t>> ranges(n_rows, std::vector<real_t>(row_len));
    for (auto& r : ranges)
        for (auto& v : r) spec >> v;
    spec >> n_s;
    if (!spec) return 2;
    std::vector<Surface*> scheme;
    int rc = 0;
    try {
        for (size_t k = 0; k < n_s; ++k) {
            int type;
            std::string tok;
            spec >> type >> tok;
            Surface* surface;
            if (type == Surface::Grating) {
                long order;
                real_t gr_const, alpha, gamma, blaze;
                size_t n_rule;
                spec >> order >> gr_const >> alpha >> gamma >> blaze >> n_rule;
                std::vector<real_t> val(n_rule);
                for (auto& v : val) spec >> v;
                if (val.size() == 1) val.insert(val.begin(), 0.0);
                if (val.empty()) val = {0.0, 1.0};
                surface = new Grating(Surface::Plane, Surface::Rectangle, Grating::Reflective,
                                      std::vector<long>(1, order), gr_const, 1.0, 1.0);
                scheme.push_back(surface);
                static_cast<Grating*>(surface)->SetRuleParams(blaze, alpha, gamma, val[0], val[1]);
            } else {
                surface = new Surface(Surface::Plane, Surface::Mirror, Surface::Circle);
                scheme.push_back(surface);
            }
            IndexSpec q = parse_index(tok);
            if (q.is_file) surface->SetQE(q.file.c_str());
            else surface->SetQE(q.value);
        }
        if (!spec) { rc = 2; throw 0; }
        FILE* file = std::fopen(out_path, "wb");
        if (!file) { rc = 2; throw 0; }
        std::vector<real_t> lambda(n_lambda, 0.0), qe_val;
        for (const auto& val : ranges) {        // scheme.cpp:1272-1334
            real_t d_lambda = (val[1] - val[0]) / (n_lambda - 1);
            for (size_t i = 0; i < n_lambda; ++i) lambda[i] = val[0] + d_lambda * i;
            qe_val = std::vector<real_t>(n_lambda, 1.0);
            size_t i_grating = 0;
            for (Surface* s : scheme) {
                switch (s->GetType()) {
                    case Surface::Grating:
                        if (ranges.size() > 1) {
                            static_cast<Grating*>(s)->SetOrder(static_cast<long>(val[i_grating + 2]));
                            ++i_grating;
                        }
                        static_cast<Grating*>(s)->ApplyQE(lambda, qe_val);
                        break;
                    case Surface::Mirror:
                    case Surface::Lens:
                        s->ApplyQE(lambda, qe_val);
                        break;
                    default:;
                }
            }
            std::fwrite(&n_lambda, sizeof(size_t), 1, file);
            std::fwrite(lambda.data(), sizeof(real_t), n_lambda, file);
            std::fwrite(qe_val.data(), sizeof(real_t), n_lambda, file);
        }
        std::fclose(file);
    } catch (Grating::bad_grating&) {
        rc = 4;
    } catch (Surface::bad_surface&) {
        rc = 3;
    } catch (TabulatedFunction::bad_tab_func& e) {
        rc = (e.bad_tab_func_error() == TabulatedFunction::OutOfRange) ? 7 : 3;
    } catch (int) {
    }
    for (Surface* s : scheme) delete s;
    return rc;
}

int main(int argc, char** argv) {
    if (argc < 2) return usage();
    rt_engine_init();
    std::string mode = argv[1];
    if (mode == "trace" && argc == 5) return run_trace(argv[2], argv[3], argv[4]);
    if (mode == "tabfunc" && argc == 5) return run_tabfunc(argv[2], argv[3], argv[4]);
    if (mode == "ccd") return run_ccd(argc, argv);
    if (mode == "qe" && argc == 4) return run_qe(argv[2], argv[3]);
    return usage();
}
