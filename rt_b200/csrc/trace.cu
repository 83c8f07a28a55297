// trace.cu -- C ABI of the device-resident engine: beam generation, the
// trace (per-surface or fused), frame counts and the reference order.
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.cuh"
#include "jit.h"
#include "rowpipe.cuh"

namespace rtb {

DevRays dev_rays(const rtb_rays* r) {
    DevRays d;
    d.X = r->X; d.Y = r->Y; d.Z = r->Z; d.cX = r->cX; d.cY = r->cY; d.cZ = r->cZ;
    d.lambda = r->lambda;
    d.flag = r->flag;
    d.lost_stage = r->lost_stage;
    d.n = r->n;
    return d;
}

// One-shot fused traces launch the kernel specialised to the scheme's
// structure when one was compiled already in this process (by a plan or
// rtb_specialize); they never compile one themselves.
int attach_compiled(PreparedScheme& ps, const rtb_trace_opts& o) {
    if (o.engine != RTB_ENGINE_FUSED ||
        (o.precision != RTB_MIXED && o.precision != RTB_MIXED32 && o.precision != RTB_FP64) || !specialize_enabled())
        return RTB_OK;
    return scheme_kernel(ps.sch, o.precision, &ps.scheme_kernel, nullptr, false);
}

int check_beams(const rtb_beam* beams, size_t n_beams, size_t n_rays, std::vector<DevBeam>& out,
                const DevScheme* sch) {
    if (!beams || n_beams == 0 || n_beams > (1u << 20)) return RTB_BAD_VALUE;
    out.resize(n_beams);
    uint64_t prev_end = 0;
    for (size_t b = 0; b < n_beams; ++b) {
        const rtb_beam& in = beams[b];
        if (in.first_ray < prev_end || in.first_ray + in.n_rays > n_rays) return RTB_BAD_VALUE;
        if (in.n_orders < 0 || in.n_orders > RTB_MAX_GRATINGS) return RTB_BAD_VALUE;
        prev_end = in.first_ray + in.n_rays;
        DevBeam& d = out[b];
        std::memset(&d, 0, sizeof(d));
        d.first_ray = in.first_ray;
        d.n_rays = in.n_rays;
        d.n_orders = in.n_orders;
        for (int g = 0; g < RTB_MAX_GRATINGS; ++g) d.orders[g] = in.orders[g];
        if (sch) beam_frame(*sch, in.center, d);
    }
    return RTB_OK;
}

FrameArgs frame_args(const rtb_trace_opts* o) {
    FrameArgs f;
    std::memset(&f, 0, sizeof(f));
    if (o->ccd && o->counts) {
        f.xsize = o->ccd->xsize;
        f.ysize = o->ccd->ysize;
        f.xpix = o->ccd->xpix;
        f.ypix = o->ccd->ypix;
        f.xdim = o->ccd->xdim;
        f.ydim = o->ccd->ydim;
        f.counts = o->counts;
        f.n_outside = reinterpret_cast<unsigned long long*>(o->n_outside);
        f.inv_xpix = 1.0 / f.xpix;
        f.inv_ypix = 1.0 / f.ypix;
    }
    return f;
}

int gen_beams(const rtb_beam* beams, size_t n_beams, size_t n_rays, std::vector<GenBeam>& gb, uint64_t* total_out) {
    if (!beams || n_beams == 0) return RTB_BAD_VALUE;
    gb.resize(n_beams);
    uint64_t prev_end = 0, total = 0;
    for (size_t b = 0; b < n_beams; ++b) {
        const rtb_beam& in = beams[b];
        if (in.shape != RTB_CIRCLE || in.n_lambda == 0 || in.first_ray < prev_end || in.first_ray + in.n_rays > n_rays)
            return RTB_BAD_VALUE;
        prev_end = in.first_ray + in.n_rays;
        total = prev_end;
        GenBeam& g = gb[b];
        g.first_ray = in.first_ray;
        g.n_rays = in.n_rays;
        g.n_lambda = in.n_lambda;
        g.seed = in.seed;
        for (int i = 0; i < 3; ++i) {
            g.disk[i] = in.disk[i];
            g.center[i] = in.center[i];
        }
        g.range[0] = in.range[0];
        g.range[1] = in.range[1];
        g.d_lambda = (in.n_lambda > 1) ? (in.range[1] - in.range[0]) / (in.n_lambda - 1) : 0.0;
        // field direction (tan fx, tan fy, 1) normalised as Beam::Normalize does
        double cx = std::tan(in.field[0]), cy = std::tan(in.field[1]), cz = 1.0;
        double acX = std::fabs(cx), acY = std::fabs(cy), acZ = std::fabs(cz), norm;
        if (acX >= acY) {
            if (acX >= acZ) norm = acX * std::sqrt(1.0 + acY * acY / acX / acX + acZ * acZ / acX / acX);
            else norm = acZ * std::sqrt(1.0 + acX * acX / acZ / acZ + acY * acY / acZ / acZ);
        } else {
            if (acY >= acZ) norm = acY * std::sqrt(1.0 + acX * acX / acY / acY + acZ * acZ / acY / acY);
            else norm = acZ * std::sqrt(1.0 + acX * acX / acZ / acZ + acY * acY / acZ / acZ);
        }
        g.c0[0] = cx / norm;
        g.c0[1] = cy / norm;
        g.c0[2] = cz / norm;
    }
    *total_out = total;
    return RTB_OK;
}

int launch_trace(const PreparedScheme& ps, TraceArgs& a, int n_beams, const rtb_trace_opts& o, const DevRays& in,
                 const DevRays& out, const FrameArgs& frame, cudaStream_t st, const uint32_t* order,
                 bool in_by_slot, const void* rows, bool out_by_slot) {
    if (o.engine == RTB_ENGINE_PER_SURFACE) {
        if (o.precision != RTB_FP64) return RTB_BAD_VALUE;
        unsigned grid = grid_for(in.n, 256, 8);
        DevRays later = out;
        later.lambda = in.lambda;  // surfaces after the first read and write `out` in place
        for (int k = 0; k < ps.sch.n_surfaces; ++k)
            k_surface_step<<<grid, 256, 0, st>>>(a.sch, k, a.knots, a.beams, n_beams, k == 0 ? in : later, out,
                                                 a.counts, a.err);
        if (frame.counts) k_ccd_frame<<<grid, 256, 0, st>>>(out, frame);
    } else if (o.engine == RTB_ENGINE_FUSED) {
        const bool m32 = o.precision == RTB_MIXED32;
        const bool mixed = o.precision == RTB_MIXED || m32;
        if (!mixed && o.precision != RTB_FP64) return RTB_BAD_VALUE;
        if (rows && !mixed) return RTB_BAD_VALUE;
        const int threads = (o.block_size > 0) ? o.block_size : 256;
        if (threads != 128 && threads != 256 && !(mixed && threads == 512)) return RTB_BAD_VALUE;
        const int rpt = (o.rays_per_thread > 0) ? o.rays_per_thread : kDefaultRpt;
        if (rpt < 1 || rpt > 64) return RTB_BAD_VALUE;
        size_t smem = fused_smem_bytes(ps.sch.n_knots);
        if (rows) smem = (smem + 127) / 128 * 128 + (m32 ? row_buffers_bytes<Row32>(threads)
                                                         : row_buffers_bytes<Row64>(threads));
        if (smem > (size_t)engine().max_smem_optin) return RTB_BAD_VALUE;
        const void* kern = ps.scheme_kernel ? ps.scheme_kernel
                           : m32           ? reinterpret_cast<const void*>(k_fused_mixed32)
                           : mixed         ? reinterpret_cast<const void*>(k_fused_mixed)
                                           : reinterpret_cast<const void*>(k_fused_fp64);
        RTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        RTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
        if (per_sm < 1) per_sm = 1;
        unsigned grid = grid_for(in.n, threads * rpt, per_sm);
        // the fused kernels' parameters, in order
        const DevScheme* sch = a.sch;
        const double* knots = a.knots;
        const DevBeam* beams = a.beams;
        int nb = n_beams;
        DevRays rin = in, rout = out;
        unsigned long long* counts = a.counts;
        unsigned* err = a.err;
        int state_out = o.state_out ? 1 : 0;
        FrameArgs fr = frame;
        TileSched ts{a.tiles, rpt, order, in_by_slot ? 1 : 0, rows, out_by_slot ? 1 : 0};
        void* params[] = {&sch, &knots, &beams, &nb, &rin, &rout, &counts, &err, &state_out, &fr, &ts};
        RTB_CUDA_TRY(cudaLaunchKernel(kern, dim3(grid), dim3(threads), params, smem, st));
    } else {
        return RTB_BAD_VALUE;
    }
    RTB_CUDA_TRY(cudaGetLastError());
    return RTB_OK;
}

int trace_result(const PreparedScheme& ps, const unsigned long long* counts, unsigned err, int n_beams,
                 rtb_trace_stats* stats) {
    const int ns = 3 * ps.sch.n_surfaces;
    uint64_t ray_surfaces = 0, n_good = 0;
    int failed_beam = -1, failed_stage = -1;
    const int total_nonaux = ps.sch.s[ps.sch.n_surfaces - 1].surfaces_upto;
    for (int b = 0; b < n_beams; ++b) {
        const unsigned long long* c = counts + (size_t)b * (ns + 1);
        uint64_t alive = c[ns];
        for (int s = 0; s < ns; ++s) alive += c[s];
        for (int s = 0; s < ns; ++s) {
            ray_surfaces += c[s] * (uint64_t)ps.sch.s[s / 3].surfaces_upto;
            if (failed_beam < 0 && c[s] > 0 && c[s] == alive) {
                failed_beam = b;
                failed_stage = s;
            }
            alive -= c[s];
        }
        ray_surfaces += c[ns] * (uint64_t)total_nonaux;
        n_good += c[ns];
    }
    if (stats) {
        stats->ray_surfaces = ray_surfaces;
        stats->n_good = n_good;
        stats->failed_beam = failed_beam;
        stats->failed_stage = failed_stage;
    }
    if (err & DEV_ERR_TIMEOUT) return RTB_FAILED;
    if (err & DEV_ERR_OUT_OF_RANGE) return RTB_OUT_OF_RANGE;
    if (err) return RTB_BAD_VALUE;
    if (failed_beam >= 0) return (failed_stage % 3 == 2) ? RTB_NO_GOOD_RAYS : RTB_NO_INTERSECTIONS;
    return RTB_OK;
}

}  // namespace rtb

using namespace rtb;

extern "C" {

int rtb_generate_beams(const rtb_beam* beams, size_t n_beams, const rtb_rays* rays, void* stream) {
    if (!rays || !beams || n_beams == 0) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    std::vector<GenBeam> gb;
    uint64_t total = 0;
    if ((st = gen_beams(beams, n_beams, rays->n, gb, &total)) != RTB_OK) return st;
    DevBuf gbuf;
    if ((st = gbuf.alloc(n_beams * sizeof(GenBeam), s)) != RTB_OK) return st;
    RTB_CUDA_TRY(cudaMemcpyAsync(gbuf.p, gb.data(), n_beams * sizeof(GenBeam), cudaMemcpyHostToDevice, s));
    DevRays dr = dev_rays(rays);
    k_generate<<<grid_for(total, 256, 8), 256, 0, s>>>(gbuf.as<GenBeam>(), (int)n_beams, total, dr);
    RTB_CUDA_TRY(cudaGetLastError());
    return RTB_OK;
}

int rtb_trace(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
              const rtb_trace_opts* opts, const rtb_rays* rays, rtb_trace_stats* stats, void* stream) {
    Range range("rtb_trace");
    if (!opts || !rays || !rays->flag || !rays->lost_stage) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    PreparedScheme ps;
    if ((st = prepare_scheme(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, ps)) != RTB_OK ||
        (st = attach_compiled(ps, *opts)) != RTB_OK)
        return st;
    std::vector<DevBeam> db;
    if ((st = check_beams(beams, n_beams, rays->n, db, &ps.sch)) != RTB_OK) return st;
    TraceArgs a;
    if ((st = a.init(ps, db, s)) != RTB_OK) return st;
    FrameArgs frame = frame_args(opts);
    DevRays dr = dev_rays(rays);
    if ((st = launch_trace(ps, a, (int)n_beams, *opts, dr, dr, frame, s)) != RTB_OK) return st;
    std::vector<unsigned long long> counts(a.counts_len);
    unsigned err = 0;
    RTB_CUDA_TRY(cudaMemcpyAsync(counts.data(), a.counts, a.counts_len * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(&err, a.err, 4, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    return trace_result(ps, counts.data(), err, (int)n_beams, stats);
}

int rtb_trace_out(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                  const rtb_trace_opts* opts, const rtb_rays* in, const rtb_rays* out, rtb_trace_stats* stats,
                  void* stream) {
    Range range("rtb_trace_out");
    if (!opts || !in || !out || !in->flag || !out->flag || !out->lost_stage || in->n != out->n) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    PreparedScheme ps;
    if ((st = prepare_scheme(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, ps)) != RTB_OK ||
        (st = attach_compiled(ps, *opts)) != RTB_OK)
        return st;
    std::vector<DevBeam> db;
    if ((st = check_beams(beams, n_beams, in->n, db, &ps.sch)) != RTB_OK) return st;
    TraceArgs a;
    if ((st = a.init(ps, db, s)) != RTB_OK) return st;
    FrameArgs frame = frame_args(opts);
    if ((st = launch_trace(ps, a, (int)n_beams, *opts, dev_rays(in), dev_rays(out), frame, s)) != RTB_OK) return st;
    std::vector<unsigned long long> counts(a.counts_len);
    unsigned err = 0;
    RTB_CUDA_TRY(cudaMemcpyAsync(counts.data(), a.counts, a.counts_len * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(&err, a.err, 4, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    return trace_result(ps, counts.data(), err, (int)n_beams, stats);
}

int rtb_ccd_frame(const rtb_rays* rays, const rtb_ccd* ccd, uint32_t* counts, uint64_t* n_outside, void* stream) {
    if (!rays || !ccd || !counts || !rays->flag) return RTB_BAD_VALUE;
    if (ccd->xdim == 0 || ccd->ydim == 0 || ccd->xdim * ccd->ydim > (1ull << 34)) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    FrameArgs f;
    f.xsize = ccd->xsize;
    f.ysize = ccd->ysize;
    f.xpix = ccd->xpix;
    f.ypix = ccd->ypix;
    f.xdim = ccd->xdim;
    f.ydim = ccd->ydim;
    f.counts = counts;
    f.n_outside = reinterpret_cast<unsigned long long*>(n_outside);
    f.inv_xpix = 1.0 / f.xpix;
    f.inv_ypix = 1.0 / f.ypix;
    k_ccd_frame<<<grid_for(rays->n, 256, 8), 256, 0, s>>>(dev_rays(rays), f);
    RTB_CUDA_TRY(cudaGetLastError());
    return RTB_OK;
}

int rtb_reference_order(const rtb_beam* beams, size_t n_beams, size_t n_stages, const rtb_rays* rays,
                        uint32_t* order, void* stream) {
    if (!rays || !rays->lost_stage || !order || n_stages > 3 * RTB_MAX_SURFACES) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    std::vector<DevBeam> db;
    if ((st = check_beams(beams, n_beams, rays->n, db)) != RTB_OK) return st;
    return reference_order(db.data(), (int)n_beams, (int)n_stages, dev_rays(rays), order, s);
}

int rtb_rearrange(size_t* n_good, double* X, double* Y, double* Z, double* cX, double* cY, double* cZ, double* lambda,
                  char* flag) {
    if (!n_good || !flag) return RTB_BAD_VALUE;
    size_t ng = *n_good;
    if (ng == 0) return RTB_OK;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = engine().stream;
    DevBuf buf;
    if ((st = buf.alloc(ng * (7 * sizeof(double) + 1), s)) != RTB_OK) return st;
    double* host[7] = {X, Y, Z, cX, cY, cZ, lambda};
    double* dev[7];
    for (int i = 0; i < 7; ++i) {
        dev[i] = buf.as<double>() + (size_t)i * ng;
        RTB_CUDA_TRY(cudaMemcpyAsync(dev[i], host[i], ng * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    char* dflag = reinterpret_cast<char*>(buf.as<double>() + 7 * ng);
    RTB_CUDA_TRY(cudaMemcpyAsync(dflag, flag, ng, cudaMemcpyHostToDevice, s));
    size_t ng_out = ng;
    if ((st = rearrange_device(ng, dev, dflag, &ng_out, s)) != RTB_OK) return st;
    for (int i = 0; i < 7; ++i)
        RTB_CUDA_TRY(cudaMemcpyAsync(host[i], dev[i], ng * sizeof(double), cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(flag, dflag, ng, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    *n_good = ng_out;
    return RTB_OK;
}

}  // extern "C"

namespace rtb {

// rtb_trace over host arrays: chunks of rays cycle through two device
// buffers on two streams, so that the copy-in of one chunk, the trace of the
// previous one and the copy-out of the one before overlap.  Page-locked host
// arrays (rtb_alocate_vector) are needed for the copies to be asynchronous.
int trace_host_impl(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                    const rtb_trace_opts* opts, const rtb_rays* h, rtb_trace_stats* stats, size_t chunk) {
    PreparedScheme ps;
    int st = prepare_scheme(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, ps);
    if (st == RTB_OK) st = attach_compiled(ps, *opts);
    if (st != RTB_OK) return st;
    std::vector<DevBeam> db;
    if ((st = check_beams(beams, n_beams, h->n, db, &ps.sch)) != RTB_OK) return st;
    const uint64_t n = h->n;
    if (n == 0) return RTB_OK;
    if (chunk == 0) chunk = (size_t)1 << 22;
    if (chunk > n) chunk = n;
    const size_t per_ray = 7 * sizeof(double) + 2;
    const int ns1 = 3 * ps.sch.n_surfaces + 1;
    cudaStream_t streams[2] = {nullptr, nullptr};
    for (auto& s : streams) RTB_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    // Per slot: device rays of one chunk, the trace arguments (scheme and
    // knots uploaded once), and page-locked staging for the chunk's beam
    // table and its counters.  Page-locked, so that no copy of a chunk blocks
    // the host and the next chunk's upload is queued while this one runs.
    struct Slot {
        DevBuf buf;
        DevRays r;
        TraceArgs args;
        DevBeam* h_beams = nullptr;
        unsigned long long* h_counts = nullptr;  // counters, then the error word
        char* h_flag = nullptr;                  // bounce buffers for pageable flag / lost_stage arrays
        uint8_t* h_lost = nullptr;
        uint64_t start = 0, cnt = 0;
        std::vector<int> beam_ids;
    };
    Slot slots[2];
    // The reference allocates Beam::flag with new[] (beam.cpp:328): a copy
    // between pageable memory and the device blocks the host, so pageable
    // flag / lost_stage arrays go through page-locked bounce buffers.
    auto pageable = [](const void* p) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            cudaGetLastError();
            return true;
        }
        return a.type == cudaMemoryTypeUnregistered;
    };
    const bool bounce_flag = pageable(h->flag);
    const bool bounce_lost = h->lost_stage && pageable(h->lost_stage);
    const size_t stage_bytes = (n_beams * sizeof(DevBeam) + (n_beams * ns1 + 1) * sizeof(unsigned long long) +
                                (bounce_flag ? chunk : 0) + (bounce_lost ? chunk : 0) + 255) / 256 * 256;
    unsigned char* h_stage = nullptr;
    if (cudaMallocHost(&h_stage, 2 * stage_bytes) != cudaSuccess) st = RTB_BAD_ALLOC;
    for (int i = 0; i < 2 && st == RTB_OK; ++i) {
        Slot& sl = slots[i];
        unsigned char* q = h_stage + i * stage_bytes;
        sl.h_beams = reinterpret_cast<DevBeam*>(q);
        q += n_beams * sizeof(DevBeam);
        sl.h_counts = reinterpret_cast<unsigned long long*>(q);
        q += (n_beams * ns1 + 1) * sizeof(unsigned long long);
        if (bounce_flag) {
            sl.h_flag = reinterpret_cast<char*>(q);
            q += chunk;
        }
        if (bounce_lost) sl.h_lost = q;
        if ((st = sl.buf.alloc(chunk * per_ray, streams[i])) != RTB_OK) break;
        if ((st = sl.args.init(ps, db, streams[i])) != RTB_OK) break;
        char* p = sl.buf.as<char>();
        double** f[7] = {&sl.r.X, &sl.r.Y, &sl.r.Z, &sl.r.cX, &sl.r.cY, &sl.r.cZ, &sl.r.lambda};
        for (int j = 0; j < 7; ++j) *f[j] = reinterpret_cast<double*>(p + (size_t)j * chunk * sizeof(double));
        sl.r.flag = reinterpret_cast<char*>(p + 7 * chunk * sizeof(double));
        sl.r.lost_stage = reinterpret_cast<uint8_t*>(p + 7 * chunk * sizeof(double) + chunk);
    }
    std::vector<unsigned long long> total((size_t)n_beams * ns1, 0);
    unsigned err_all = 0;
    FrameArgs frame = frame_args(opts);
    rtb_trace_opts o = *opts;
    o.engine = RTB_ENGINE_FUSED;
    double* hin[7] = {h->X, h->Y, h->Z, h->cX, h->cY, h->cZ, h->lambda};
    auto drain = [&](Slot& sl, cudaStream_t s) -> int {
        RTB_CUDA_TRY(cudaStreamSynchronize(s));
        const size_t nb = sl.beam_ids.size();
        for (size_t b = 0; b < nb; ++b)
            for (int k = 0; k < ns1; ++k) total[(size_t)sl.beam_ids[b] * ns1 + k] += sl.h_counts[b * ns1 + k];
        err_all |= (unsigned)(sl.h_counts[nb * ns1] & 0xffffffffu);
        if (sl.h_flag) std::memcpy(h->flag + sl.start, sl.h_flag, sl.cnt);
        if (sl.h_lost) std::memcpy(h->lost_stage + sl.start, sl.h_lost, sl.cnt);
        sl.beam_ids.clear();
        return RTB_OK;
    };
    uint64_t start = 0;
    int it = 0;
    while (st == RTB_OK && start < n) {
        Slot& sl = slots[it & 1];
        cudaStream_t s = streams[it & 1];
        if (!sl.beam_ids.empty() && (st = drain(sl, s)) != RTB_OK) break;
        uint64_t cnt = (n - start < chunk) ? n - start : chunk;
        // beams overlapping [start, start+cnt), rebased to the chunk
        size_t nb = 0;
        for (size_t b = 0; b < n_beams; ++b) {
            uint64_t a0 = db[b].first_ray, a1 = db[b].first_ray + db[b].n_rays;
            uint64_t lo = a0 > start ? a0 : start, hi = a1 < start + cnt ? a1 : start + cnt;
            if (lo >= hi) continue;
            DevBeam d = db[b];
            d.first_ray = lo - start;
            d.n_rays = hi - lo;
            sl.h_beams[nb++] = d;
            sl.beam_ids.push_back((int)b);
        }
        if (nb == 0) {  // rays outside every beam are not traced
            start += cnt;
            ++it;
            continue;
        }
        sl.r.n = cnt;
        sl.start = start;
        sl.cnt = cnt;
        for (int j = 0; j < 7; ++j)
            RTB_CUDA_TRY(cudaMemcpyAsync((&sl.r.X)[j], hin[j] + start, cnt * sizeof(double), cudaMemcpyHostToDevice, s));
        const char* flag_src = h->flag + start;
        if (sl.h_flag) {
            std::memcpy(sl.h_flag, flag_src, cnt);
            flag_src = sl.h_flag;
        }
        RTB_CUDA_TRY(cudaMemcpyAsync(sl.r.flag, flag_src, cnt, cudaMemcpyHostToDevice, s));
        if (h->lost_stage) {
            const uint8_t* lost_src = h->lost_stage + start;
            if (sl.h_lost) {
                std::memcpy(sl.h_lost, lost_src, cnt);
                lost_src = sl.h_lost;
            }
            RTB_CUDA_TRY(cudaMemcpyAsync(sl.r.lost_stage, lost_src, cnt, cudaMemcpyHostToDevice, s));
        } else
            RTB_CUDA_TRY(cudaMemsetAsync(sl.r.lost_stage, RTB_NOT_LOST, cnt, s));
        RTB_CUDA_TRY(cudaMemcpyAsync(sl.args.beams, sl.h_beams, nb * sizeof(DevBeam), cudaMemcpyHostToDevice, s));
        sl.args.counts_len = nb * ns1;
        RTB_CUDA_TRY(cudaMemsetAsync(sl.args.counts, 0, sl.args.counts_len * 8, s));
        RTB_CUDA_TRY(cudaMemsetAsync(sl.args.err, 0, 256, s));  // error word and tile counter
        if ((st = launch_trace(ps, sl.args, (int)nb, o, sl.r, sl.r, frame, s)) != RTB_OK) break;
        int nout = o.state_out ? 6 : 2;
        for (int j = 0; j < nout; ++j)
            RTB_CUDA_TRY(cudaMemcpyAsync(hin[j] + start, (&sl.r.X)[j], cnt * sizeof(double), cudaMemcpyDeviceToHost, s));
        RTB_CUDA_TRY(cudaMemcpyAsync(sl.h_flag ? sl.h_flag : h->flag + start, sl.r.flag, cnt, cudaMemcpyDeviceToHost, s));
        if (h->lost_stage)
            RTB_CUDA_TRY(cudaMemcpyAsync(sl.h_lost ? sl.h_lost : h->lost_stage + start, sl.r.lost_stage, cnt,
                                         cudaMemcpyDeviceToHost, s));
        RTB_CUDA_TRY(cudaMemcpyAsync(sl.h_counts, sl.args.counts, sl.args.counts_len * 8, cudaMemcpyDeviceToHost, s));
        RTB_CUDA_TRY(cudaMemcpyAsync(sl.h_counts + sl.args.counts_len, sl.args.err, 4, cudaMemcpyDeviceToHost, s));
        start += cnt;
        ++it;
    }
    for (int i = 0; i < 2; ++i) {
        if (!slots[i].beam_ids.empty()) {
            int s2 = drain(slots[i], streams[i]);
            if (st == RTB_OK) st = s2;
        }
        if (streams[i]) cudaStreamSynchronize(streams[i]);
    }
    for (int i = 0; i < 2; ++i) {
        slots[i].args.buf.release();
        slots[i].buf.release();
    }
    for (auto& s : streams) {
        if (!s) continue;
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    if (h_stage) cudaFreeHost(h_stage);
    if (st != RTB_OK) return st;
    return trace_result(ps, total.data(), err_all, (int)n_beams, stats);
}

}  // namespace rtb

extern "C" RTB_API int rtb_trace_host(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams,
                                      size_t n_beams, const rtb_trace_opts* opts, const rtb_rays* host_rays,
                                      rtb_trace_stats* stats) {
    Range range("rtb_trace_host");
    if (!opts || !host_rays || !host_rays->flag) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    return trace_host_impl(surfaces, n_surfaces, beams, n_beams, opts, host_rays, stats, 0);
}
