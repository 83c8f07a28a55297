// noalloc.cu -- the fused trace for callers that cannot allocate memory.
//
// rtb_trace_out allocates per call (stream-ordered pool) the scratch that
// its fused kernel reads: the prepared scheme, the knot tables, the beam table,
// the per-(beam, stage) loss counters and an error word.  Some callers cannot
// let a library allocate: applications whose own allocator has reserved the
// device memory up front, or code running with a fixed memory budget where no
// allocator may be called once it has started.  rtb_trace_out_noalloc runs the
// same fused kernels (k_fused_fp64 / k_fused_mixed, unchanged) with that
// scratch in the file-scope device array below, and stages the host side of it
// in file-scope host arrays: no cudaMalloc, cudaFree, pool allocation or heap
// allocation.
//
// Limits: RTB_NOALLOC_SCRATCH_BYTES (1 MiB) of device scratch per device,
// which holds the scheme (<= RTB_MAX_SURFACES surfaces), up to
// RTB_NOALLOC_MAX_KNOTS table values, the beam table and n_beams *
// (3 * n_surfaces + 1) loss counters; requests that do not fit, or whose
// launch needs more shared memory than a block may have, return
// RTB_BAD_VALUE before any work is queued.  With the largest tables the
// counters leave room for 1,100 beams of a 32-surface scheme.
//
// The array is set up once per device, on the first call made with that
// device current (cudaGetSymbolAddress).  Every call on a device shares the
// array and leaves its contents behind; each call clears the counters it
// uses.  Calls run one at a time (the engine lock) and each returns with its
// stream synchronised, so calls of this library do not overlap on the GPU;
// other work that writes the array while a call runs would race with it.
#include <cstring>

#include "engine.cuh"

namespace rtb {

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[RTB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Host-side staging of the scratch contents (no heap).
alignas(256) unsigned char h_stage[RTB_NOALLOC_SCRATCH_BYTES];
DevScheme h_scheme;

struct Layout {
    size_t knots, beams, counts, err, total;
};

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

Layout layout(size_t n_knots, size_t n_beams, size_t n_counts) {
    Layout l;
    l.knots = align256(sizeof(DevScheme));
    l.beams = l.knots + align256(n_knots * sizeof(double));
    l.counts = l.beams + align256(n_beams * sizeof(DevBeam));
    l.err = l.counts + align256(n_counts * sizeof(unsigned long long));
    l.total = l.err + 256;
    return l;
}

// Device address of the scratch array on the current device (set up once).
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RTB_FAILED;
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RTB_FAILED;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return RTB_OK;
}

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" RTB_API int rtb_trace_out_noalloc(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams,
                                             size_t n_beams, const rtb_trace_opts* opts, const rtb_rays* in,
                                             const rtb_rays* out, rtb_trace_stats* stats, void* stream) {
    if (!opts || !in || !out || !in->flag || !out->flag || !out->lost_stage || in->n != out->n) return RTB_BAD_VALUE;
    if (opts->engine != RTB_ENGINE_FUSED) return RTB_BAD_VALUE;
    if (opts->precision != RTB_FP64 && opts->precision != RTB_MIXED) return RTB_BAD_VALUE;
    if (!beams || n_beams == 0 || n_surfaces == 0 || n_surfaces > RTB_MAX_SURFACES) return RTB_BAD_VALUE;
    const bool mixed = opts->precision == RTB_MIXED;
    // the launch configuration rtb_trace_out accepts (launch_trace)
    const int threads = (opts->block_size > 0) ? opts->block_size : 256;
    if (threads != 128 && threads != 256 && !(mixed && threads == 512)) return RTB_BAD_VALUE;
    const int rpt = (opts->rays_per_thread > 0) ? opts->rays_per_thread : kDefaultRpt;
    if (rpt < 1 || rpt > 64) return RTB_BAD_VALUE;
    const size_t ns1 = 3 * n_surfaces + 1;
    if (layout(0, n_beams, n_beams * ns1).total > RTB_NOALLOC_SCRATCH_BYTES) return RTB_BAD_VALUE;
    std::lock_guard<std::mutex> lock(engine().mu);
    int st = ensure_init();
    if (st != RTB_OK) return st;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return RTB_FAILED;
    // the library's own stream belongs to the device it was set up on
    if (!stream && dev != engine().device) return RTB_BAD_VALUE;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;

    // everything is prepared and checked in the host staging before the
    // first copy is queued: the scheme by the same code as every other trace
    // (prepare_scheme_into), its tables packed at their final offset
    const size_t knots_at = layout(0, 0, 0).knots;
    KnotBuf kb(reinterpret_cast<double*>(h_stage + knots_at), RTB_NOALLOC_MAX_KNOTS);
    if ((st = prepare_scheme_into(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, h_scheme, kb)) !=
        RTB_OK)
        return st;
    const size_t n_knots = kb.size();
    const Layout l = layout(n_knots, n_beams, n_beams * ns1);
    if (l.total > RTB_NOALLOC_SCRATCH_BYTES) return RTB_BAD_VALUE;
    const size_t smem = fused_smem_bytes((int)n_knots);
    if (smem > (size_t)engine().max_smem_optin) return RTB_BAD_VALUE;
    std::memcpy(h_stage, &h_scheme, sizeof(DevScheme));
    DevBeam* beams_h = reinterpret_cast<DevBeam*>(h_stage + l.beams);
    uint64_t prev_end = 0;
    for (size_t b = 0; b < n_beams; ++b) {
        const rtb_beam& bi = beams[b];
        if (bi.first_ray < prev_end || bi.first_ray + bi.n_rays > in->n) return RTB_BAD_VALUE;
        if (bi.n_orders < 0 || bi.n_orders > RTB_MAX_GRATINGS) return RTB_BAD_VALUE;
        prev_end = bi.first_ray + bi.n_rays;
        std::memset(&beams_h[b], 0, sizeof(DevBeam));
        beams_h[b].first_ray = bi.first_ray;
        beams_h[b].n_rays = bi.n_rays;
        beams_h[b].n_orders = bi.n_orders;
        for (int g = 0; g < RTB_MAX_GRATINGS; ++g) beams_h[b].orders[g] = bi.orders[g];
    }
    auto kern = mixed ? k_fused_mixed : k_fused_fp64;
    RTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    if (per_sm < 1) per_sm = 1;
    void* base = nullptr;
    if ((st = scratch_address(&base)) != RTB_OK) return st;

    unsigned char* d = static_cast<unsigned char*>(base);
    RTB_CUDA_TRY(cudaMemcpyAsync(d, h_stage, l.counts, cudaMemcpyHostToDevice, s));
    RTB_CUDA_TRY(cudaMemsetAsync(d + l.counts, 0, l.total - l.counts, s));
    FrameArgs frame;
    std::memset(&frame, 0, sizeof(frame));
    if (opts->ccd && opts->counts) {
        frame.xsize = opts->ccd->xsize;
        frame.ysize = opts->ccd->ysize;
        frame.xpix = opts->ccd->xpix;
        frame.ypix = opts->ccd->ypix;
        frame.xdim = opts->ccd->xdim;
        frame.ydim = opts->ccd->ydim;
        frame.counts = opts->counts;
        frame.n_outside = reinterpret_cast<unsigned long long*>(opts->n_outside);
        frame.inv_xpix = 1.0 / frame.xpix;
        frame.inv_ypix = 1.0 / frame.ypix;
    }
    DevRays ri, ro;
    ri.X = in->X; ri.Y = in->Y; ri.Z = in->Z; ri.cX = in->cX; ri.cY = in->cY; ri.cZ = in->cZ;
    ri.lambda = in->lambda; ri.flag = in->flag; ri.lost_stage = in->lost_stage; ri.n = in->n;
    ro.X = out->X; ro.Y = out->Y; ro.Z = out->Z; ro.cX = out->cX; ro.cY = out->cY; ro.cZ = out->cZ;
    ro.lambda = out->lambda; ro.flag = out->flag; ro.lost_stage = out->lost_stage; ro.n = out->n;
    unsigned long long* counts_d = reinterpret_cast<unsigned long long*>(d + l.counts);
    unsigned* err_d = reinterpret_cast<unsigned*>(d + l.err);
    // the tile counter shares the zeroed 256-byte error slot
    unsigned long long* tiles_d = reinterpret_cast<unsigned long long*>(d + l.err + 64);
    kern<<<grid_for(in->n, threads * rpt, per_sm), threads, smem, s>>>(
        reinterpret_cast<const DevScheme*>(d), reinterpret_cast<const double*>(d + l.knots),
        reinterpret_cast<const DevBeam*>(d + l.beams), (int)n_beams, ri, ro, counts_d, err_d,
        opts->state_out ? 1 : 0, frame, TileSched{tiles_d, rpt, nullptr, 0});
    RTB_CUDA_TRY(cudaGetLastError());
    unsigned long long* counts_h = reinterpret_cast<unsigned long long*>(h_stage + l.counts);
    unsigned err = 0;
    RTB_CUDA_TRY(cudaMemcpyAsync(counts_h, counts_d, n_beams * ns1 * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(&err, err_d, 4, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));

    // status and statistics, as trace_result() derives them
    const int ns = 3 * (int)n_surfaces;
    const int total_nonaux = h_scheme.s[n_surfaces - 1].surfaces_upto;
    uint64_t ray_surfaces = 0, n_good = 0;
    int failed_beam = -1, failed_stage = -1;
    for (size_t b = 0; b < n_beams; ++b) {
        const unsigned long long* c = counts_h + b * ns1;
        uint64_t alive = c[ns];
        for (int k = 0; k < ns; ++k) alive += c[k];
        for (int k = 0; k < ns; ++k) {
            ray_surfaces += c[k] * (uint64_t)h_scheme.s[k / 3].surfaces_upto;
            if (failed_beam < 0 && c[k] > 0 && c[k] == alive) {
                failed_beam = (int)b;
                failed_stage = k;
            }
            alive -= c[k];
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
    if (err & DEV_ERR_OUT_OF_RANGE) return RTB_OUT_OF_RANGE;
    if (err) return RTB_BAD_VALUE;
    if (failed_beam >= 0) return (failed_stage % 3 == 2) ? RTB_NO_GOOD_RAYS : RTB_NO_INTERSECTIONS;
    return RTB_OK;
}
