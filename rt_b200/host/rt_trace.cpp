// rt_trace -- the reference's ray-tracing program (ray-tracing/main.cpp with
// Scheme::run, common-lib/scheme.cpp:878-1099) on the B200 engine.
//
//   rt_trace scheme_file rt_files_file [log_file] [--precision fp64|mixed|mixed32]
//            [--fixes N] [--seed S] [--bench K]
//
// Loads the scheme file (rtb_scheme_load), writes the input beam as
// <result_file>_input_beam.dat, traces every wavelength range -- one range,
// or one per row of the range file, whose columns after the two wavelengths
// are the gratings' orders -- and writes each result as
// <result_file>_range_(w1-w2).dat (several ranges) or <result_file>.dat (one),
// good rays first, in the order the reference's Rearrange calls leave them.
// The names of the result files go to rt_files_file, one per line.
//
// The beams are the reference's PARALLEL circular beams with RANDOM profile
// (uniform on the disk R_in..R_out) and UNIFORM (composite with <nlambda>, or
// one wavelength per ray) or MONOCHROMATIC wavelengths.  The reference seeds
// its generator from the clock (cuda_engine/rt_cuda_engine_beam.cu:270-275);
// here every range draws its positions from Philox4x32-10 keyed by
// seed + range index, so a run can be repeated.  The engine is the fused FP64
// kernel by default (the same bits as the reference's per-surface loop on the
// CPU oracle); --precision mixed selects the mixed-precision kernel (FP64
// ray state), mixed32 the one with FP32 ray state.
//
// --bench K times the trace instead of writing results: every range becomes
// one beam of a plan (rtb_plan_*: rays generated on the device, coherent
// tracing order, outputs at the tracing slots, launch configuration from the
// autotuner), and K plan runs are timed with CUDA events on the plan's stream,
// after three untimed ones; the program prints ms per run and ray-surfaces
// per second.  This timing goes through the C ABI alone.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "rtb.h"

namespace {

struct DeviceRays {
    std::vector<void*> mem;
    rtb_rays r{};
    bool alloc(size_t n) {
        double** f[7] = {&r.X, &r.Y, &r.Z, &r.cX, &r.cY, &r.cZ, &r.lambda};
        for (auto p : f) {
            void* q = nullptr;
            if (cudaMalloc(&q, n * sizeof(double)) != cudaSuccess) return false;
            mem.push_back(q);
            *p = static_cast<double*>(q);
        }
        void* q = nullptr;
        if (cudaMalloc(&q, 2 * n + 16) != cudaSuccess) return false;
        mem.push_back(q);
        r.flag = static_cast<char*>(q);
        r.lost_stage = reinterpret_cast<uint8_t*>(static_cast<char*>(q) + n + 16);
        r.n = n;
        return true;
    }
    ~DeviceRays() {
        for (void* p : mem) cudaFree(p);
    }
};

int fail(const char* what, int code = 1) {
    std::fprintf(stderr, "rt_trace: %s\n", what);
    return code;
}

const char* scheme_error_text(int e) {
    static const char* t[] = {"Can not open scheme file!",
                              "A parsing error occured while loading scheme file!",
                              "No class attribute!",
                              "Bad attribute in the input scheme file!",
                              "Not a number attribute!",
                              "Memory allocation error occured while parsing input scheme!",
                              "There was no general scheme description in the input scheme file!",
                              "There was no beam description in the input scheme file!",
                              "No one surface description was found in the input scheme file!",
                              "There was neither range attrribute or range file in the input scheme file!",
                              "Can not find range file!",
                              "Bad range value!"};
    return (e >= 0 && e < (int)(sizeof(t) / sizeof(t[0]))) ? t[e] : "Unknown scheme error!";
}

}  // namespace

// --bench: every range one beam of a plan, K timed runs.
int run_bench(const rtb_surface* surf, size_t ns, size_t n_rows, int K, int precision, uint32_t fixes,
              uint64_t seed, uint64_t n_per, uint64_t n_lambda, uint64_t n_rays, const rtb_scheme_beam& bd,
              const double* rows, size_t row_len, int n_gratings) {
    std::vector<rtb_beam> beams(n_rows);
    for (size_t r = 0; r < n_rows; ++r) {
        rtb_beam& b = beams[r];
        std::memset(&b, 0, sizeof(b));
        b.first_ray = r * n_rays;
        b.n_rays = n_rays;
        b.shape = RTB_CIRCLE;
        b.disk[0] = (double)n_per;
        b.disk[1] = bd.params[1];
        b.disk[2] = bd.params[2];
        for (int i = 0; i < 3; ++i) b.center[i] = bd.center[i];
        const double* row = rows + r * row_len;
        b.range[0] = row[0];
        b.range[1] = (bd.range_distr == RTB_RANGE_MONOCHROMATIC) ? row[0] : row[1];
        b.n_lambda = n_lambda;
        b.seed = seed + r;
        if (n_rows > 1 && (int)row_len >= 2 + n_gratings) {
            b.n_orders = n_gratings;
            for (int g = 0; g < n_gratings && g < RTB_MAX_GRATINGS; ++g) b.orders[g] = (int64_t)row[2 + g];
        }
    }
    rtb_trace_opts o;
    std::memset(&o, 0, sizeof(o));
    o.engine = RTB_ENGINE_FUSED;
    o.precision = precision;
    o.fixes = fixes;
    o.renormalize_lost = 1;
    o.state_out = 0;
    o.out_order = RTB_OUT_SLOT;
    rtb_plan* plan = nullptr;
    int st = rtb_plan_create(surf, ns, beams.data(), beams.size(), &o, &plan);
    if (st != RTB_OK) return fail("plan creation failed", 2);
    rtb_tune_entry tune[16];
    size_t n_tune = 0;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rtb_plan_autotune(plan, 2, tune, 16, &n_tune) != RTB_OK ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        rtb_plan_destroy(plan);
        return fail("bench set-up failed", 2);
    }
    int rc = 0;
    for (int i = 0; i < 3 && !rc; ++i) rc = rtb_plan_run(plan, s) != RTB_OK;
    cudaEventRecord(e0, s);
    for (int i = 0; i < K && !rc; ++i) rc = rtb_plan_run(plan, s) != RTB_OK;
    cudaEventRecord(e1, s);
    float ms = 0.f;
    rtb_trace_stats stats;
    if (!rc && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)) rc = 1;
    const int rs = rc ? RTB_FAILED : rtb_plan_result(plan, &stats);
    int32_t block = 0, rpt = 0;
    uint64_t n = 0;
    rtb_plan_config(plan, &block, &rpt, &n);
    int32_t spec = 0;
    rtb_plan_specialized(plan, &spec, nullptr, 0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    rtb_plan_destroy(plan);
    if (rc || (rs != RTB_OK && rs != RTB_NO_INTERSECTIONS && rs != RTB_NO_GOOD_RAYS))
        return fail("bench run failed", 2);
    const double per = (double)ms / K;
    std::printf("rt_trace bench: %llu rays in %zu ranges, %llu ray-surfaces and %llu good rays per run; "
                "%s kernel%s, block %d x %d rays per thread; %.4f ms per run, %.4g ray-surfaces/s\n",
                (unsigned long long)n, n_rows, (unsigned long long)stats.ray_surfaces,
                (unsigned long long)stats.n_good,
                precision == RTB_FP64 ? "fused FP64" : (precision == RTB_MIXED ? "fused mixed" : "fused mixed32"),
                spec ? " (specialised)" : "", block, rpt, per, (double)stats.ray_surfaces / (per * 1e-3));
    return 0;
}

int main(int argc, char** argv) {
    std::vector<std::string> pos;
    int precision = RTB_FP64;
    uint32_t fixes = 0;
    uint64_t seed = 20141203;
    int bench = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--precision" && i + 1 < argc) {
            std::string v = argv[++i];
            if (v == "mixed") precision = RTB_MIXED;
            else if (v == "mixed32") precision = RTB_MIXED32;
            else if (v != "fp64") return fail("--precision is fp64, mixed or mixed32");
        } else if (a == "--bench" && i + 1 < argc) {
            bench = std::atoi(argv[++i]);
            if (bench < 1) return fail("--bench takes a number of runs");
        } else if (a == "--fixes" && i + 1 < argc) {
            fixes = (uint32_t)std::strtoul(argv[++i], nullptr, 0);
        } else if (a == "--seed" && i + 1 < argc) {
            seed = std::strtoull(argv[++i], nullptr, 0);
        } else {
            pos.push_back(a);
        }
    }
    if (pos.size() < 2) {
        std::fprintf(stderr, "Usage: rt_trace scheme_filename rt_files_filename [log_file] "
                             "[--precision fp64|mixed|mixed32] [--fixes N] [--seed S] [--bench K]\n");
        return 1;
    }
    std::ofstream logf;
    if (pos.size() > 2) logf.open(pos[2]);
    std::ostream& log = logf.is_open() ? static_cast<std::ostream&>(logf) : std::cout;

    std::printf("Loading scheme file ... ");
    rtb_scheme* sc = nullptr;
    int serr = -1;
    if (rtb_scheme_load(pos[0].c_str(), &sc, &serr) != RTB_OK) {
        std::printf("\n");
        return fail(scheme_error_text(serr));
    }
    std::printf("OK!\n");
    const rtb_surface* surf = nullptr;
    size_t ns = 0;
    rtb_scheme_surfaces(sc, &surf, &ns);
    std::printf("Loaded %zu surfaces.\n", ns);
    rtb_scheme_beam bd;
    rtb_scheme_get_beam(sc, &bd);
    const double* rows = nullptr;
    size_t n_rows = 0, row_len = 0;
    rtb_scheme_ranges(sc, &rows, &n_rows, &row_len);
    if (bd.type != RTB_BEAM_PARALLEL || bd.shape != RTB_CIRCLE || bd.profile != RTB_PROFILE_RANDOM ||
        bd.range_distr == RTB_RANGE_RANDOM || bd.n_params < 3) {
        rtb_scheme_free(sc);
        return fail("only PARALLEL circular beams with RANDOM profile and UNIFORM or MONOCHROMATIC "
                    "wavelengths are generated on the device");
    }
    const uint64_t n_per = (uint64_t)bd.params[0];
    uint64_t n_lambda = 1, n_rays = n_per;
    if (bd.range_distr == RTB_RANGE_UNIFORM) {
        n_lambda = bd.n_lambda ? bd.n_lambda : n_per;  // composite, or one wavelength per ray
        n_rays = bd.n_lambda ? n_per * bd.n_lambda : n_per;
    }
    int n_gratings = 0;
    for (size_t k = 0; k < ns; ++k) n_gratings += surf[k].type == RTB_GRATING;

    if (bench > 0) {
        const int rc = run_bench(surf, ns, n_rows, bench, precision, fixes, seed, n_per, n_lambda, n_rays, bd, rows,
                                 row_len, n_gratings);
        rtb_scheme_free(sc);
        return rc;
    }
    DeviceRays rays;
    uint32_t* order = nullptr;
    if (!rays.alloc(n_rays) || cudaMalloc(&order, n_rays * sizeof(uint32_t)) != cudaSuccess) {
        rtb_scheme_free(sc);
        return fail("device memory");
    }
    const std::string root = rtb_scheme_text(sc, RTB_SCHEME_RESULT_FILE);
    char info[512] = {0};
    rtb_info(info, sizeof(info));
    log << "\nRAY-TRACING ON B200\n\n  ENGINE INFO:\n    " << info << "\n\n  The scheme was loaded from: " << pos[0]
        << "\n  Scheme description: " << rtb_scheme_text(sc, RTB_SCHEME_NAME) << "\n";

    auto beam_for = [&](size_t r) {
        rtb_beam b;
        std::memset(&b, 0, sizeof(b));
        b.first_ray = 0;
        b.n_rays = n_rays;
        b.shape = RTB_CIRCLE;
        b.disk[0] = (double)n_per;
        b.disk[1] = bd.params[1];
        b.disk[2] = bd.params[2];
        for (int i = 0; i < 3; ++i) b.center[i] = bd.center[i];
        const double* row = rows + r * row_len;
        b.range[0] = row[0];
        b.range[1] = (bd.range_distr == RTB_RANGE_MONOCHROMATIC) ? row[0] : row[1];
        b.n_lambda = n_lambda;
        b.seed = seed + r;
        if (n_rows > 1 && (int)row_len >= 2 + n_gratings) {  // orders from the range file (scheme.cpp:1026-1032)
            b.n_orders = n_gratings;
            for (int g = 0; g < n_gratings && g < RTB_MAX_GRATINGS; ++g) b.orders[g] = (int64_t)row[2 + g];
        }
        return b;
    };

    int rc = 0;
    std::vector<std::string> results;
    rtb_trace_opts o;
    std::memset(&o, 0, sizeof(o));
    o.engine = RTB_ENGINE_FUSED;
    o.precision = precision;
    o.fixes = fixes;
    o.renormalize_lost = 1;
    o.state_out = 1;
    std::printf("Run ... ");
    std::fflush(stdout);
    {
        rtb_beam b0 = beam_for(0);
        if (rtb_generate_beams(&b0, 1, &rays.r, nullptr) != RTB_OK) rc = fail("beam generation");
        // the input beam: every ray good, in generation order
        std::vector<uint32_t> ident(n_rays);
        for (uint64_t k = 0; k < n_rays; ++k) ident[k] = (uint32_t)k;
        if (!rc && cudaMemcpy(order, ident.data(), n_rays * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail("copy");
        if (!rc && rtb_save_dat((root + "_input_beam.dat").c_str(), &rays.r, order, 0, n_rays, n_rays, n_lambda,
                                nullptr) != RTB_OK)
            rc = fail("cannot write the input beam");
    }
    log << "\n  Number of wavelength ranges: " << n_rows << "\n\n  Total number of rays in beam: " << n_rays << "\n";
    for (size_t r = 0; r < n_rows && !rc; ++r) {
        const double* row = rows + r * row_len;
        log << "\n  *** Current range: [" << row[0] << "," << row[1] << "] ***\n";
        rtb_beam b = beam_for(r);
        if (rtb_generate_beams(&b, 1, &rays.r, nullptr) != RTB_OK) {
            rc = fail("beam generation");
            break;
        }
        rtb_trace_stats st;
        int t = rtb_trace(surf, ns, &b, 1, &o, &rays.r, &st, nullptr);
        if (t != RTB_OK) {  // the reference's Scheme::run throws here
            log << "ERROR!\n";
            std::fprintf(stderr, "rt_trace: range %zu: status %d (first failing stage %d)\n", r, t,
                         st.failed_stage);
            rc = 2;
            break;
        }
        log << "    good rays at the end: " << st.n_good << " (" << st.ray_surfaces << " ray-surfaces)\n";
        if (rtb_reference_order(&b, 1, 3 * ns, &rays.r, order, nullptr) != RTB_OK) {
            rc = fail("order");
            break;
        }
        std::ostringstream fn;
        if (n_rows > 1) fn << root << "_range_(" << row[0] << "-" << row[1] << ").dat";
        else fn << root << ".dat";
        if (rtb_save_dat(fn.str().c_str(), &rays.r, order, 0, n_rays, st.n_good, n_lambda, nullptr) != RTB_OK) {
            rc = fail("cannot write a result file");
            break;
        }
        results.push_back(fn.str());
    }
    if (!rc) {
        std::printf("OK!\n");
        std::ofstream lst(pos[1]);
        for (const auto& s : results) lst << s << "\n";
    }
    cudaFree(order);
    rtb_scheme_free(sc);
    return rc;
}
