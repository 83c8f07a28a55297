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
// RTB_NOALLOC_MAX_KNOTS table values, and n_beams * (3 * n_surfaces + 1) loss
// counters plus the beam table; larger requests return RTB_BAD_VALUE before
// any work is queued.
//
// The array is set up once per device, on the first call made with that
// device current (cudaGetSymbolAddress); that first call should come before any
// stream capture.  Every call on a device shares the array and leaves its
// contents behind; each call clears the counters it uses.  Calls that overlap
// on the GPU (concurrent streams, or a second call issued from another thread
// before the first has returned) race on the array.
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

// A table appended to a fixed buffer, laid out as add_table() lays it out.
int put_table(const rtb_table* t, double* knots, size_t cap, size_t& used, int32_t& off, int32_t& cnt) {
    if (!t || t->n == 0 || !t->y) return RTB_BAD_VALUE;
    size_t need = (t->n == 1) ? 3 : 3 * t->n;
    if (t->n != 1 && (t->n < 4 || t->n > RTB_MAX_KNOTS || !t->x || !t->y2)) return RTB_BAD_VALUE;
    if (used + need > cap) return RTB_BAD_VALUE;
    off = (int32_t)used;
    if (t->n == 1) {
        cnt = 1;
        knots[used] = 0.0;
        knots[used + 1] = t->y[0];
        knots[used + 2] = 0.0;
    } else {
        cnt = (int32_t)t->n;
        std::memcpy(knots + used, t->x, t->n * sizeof(double));
        std::memcpy(knots + used + t->n, t->y, t->n * sizeof(double));
        std::memcpy(knots + used + 2 * t->n, t->y2, t->n * sizeof(double));
    }
    used += need;
    return RTB_OK;
}

// The scheme preparation of prepare_scheme() into fixed buffers.
int prepare_fixed(const rtb_surface* surf, size_t n, uint32_t fixes, int renorm_lost, DevScheme& out, double* knots,
                  size_t cap, size_t& n_knots) {
    if (!surf || n == 0 || n > RTB_MAX_SURFACES) return RTB_BAD_VALUE;
    std::memset(&out, 0, sizeof(out));
    n_knots = 0;
    int32_t o, c;
    rtb_table unit = {1, nullptr, nullptr, nullptr};
    double one = 1.0;
    unit.y = &one;
    if (put_table(&unit, knots, cap, n_knots, o, c) != RTB_OK) return RTB_BAD_VALUE;
    int ng = 0, nonaux = 0;
    for (size_t k = 0; k < n; ++k) {
        const rtb_surface& in = surf[k];
        DevSurface& s = out.s[k];
        bool non_aux = in.type != RTB_AUX_TYPE;
        int st = surface_from_params(non_aux ? in.cls : RTB_AUX_CLASS, in.params, s);
        if (st != RTB_OK) return st;
        if (in.type < RTB_MIRROR || in.type > RTB_AUX_TYPE) return RTB_BAD_VALUE;
        if (in.shape != RTB_CIRCLE && in.shape != RTB_RECTANGLE) return RTB_BAD_VALUE;
        if (in.type == RTB_GRATING && in.grating_type != RTB_REFLECTIVE && in.grating_type != RTB_TRANSPARENT)
            return RTB_BAD_VALUE;
        s.cls = in.cls;
        s.type = in.type;
        s.shape = in.shape;
        s.gr_type = in.grating_type;
        s.non_aux = non_aux;
        if (!non_aux) s.kind = IS_NONE;
        s.order = in.order;
        s.gr_const = in.gr_const;
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
            if ((st = put_table(&in.n2, knots, cap, n_knots, s.n2_off, s.n2_n)) != RTB_OK) return st;
            if (in.type == RTB_LENS || in.grating_type == RTB_TRANSPARENT)
                if ((st = put_table(&in.n1, knots, cap, n_knots, s.n1_off, s.n1_n)) != RTB_OK) return st;
        }
        s.grating_index = (s.type == RTB_GRATING) ? ng++ : -1;
        if (s.non_aux) ++nonaux;
        s.surfaces_upto = nonaux;
    }
    if (ng > RTB_MAX_GRATINGS) return RTB_BAD_VALUE;
    for (size_t k = 0; k < n; ++k) {
        int cnt = out.s[k].non_aux ? 1 : 0;
        for (size_t j = k + 1; j < n; ++j) cnt += 1 + (out.s[j].non_aux ? 1 : 0);
        out.s[k].renorm_after = cnt;
    }
    out.n_surfaces = (int32_t)n;
    out.n_knots = (int32_t)n_knots;
    out.fixes = fixes;
    out.renorm_lost = renorm_lost;
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
    const size_t ns1 = 3 * n_surfaces + 1;
    // size checks before anything is written
    {
        Layout worst = layout(RTB_NOALLOC_MAX_KNOTS, n_beams, n_beams * ns1);
        if (worst.total > RTB_NOALLOC_SCRATCH_BYTES) return RTB_BAD_VALUE;
    }
    std::lock_guard<std::mutex> lock(engine().mu);
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    void* base = nullptr;
    if ((st = scratch_address(&base)) != RTB_OK) return st;

    Layout l0 = layout(RTB_NOALLOC_MAX_KNOTS, n_beams, n_beams * ns1);
    double* knots_h = reinterpret_cast<double*>(h_stage + l0.knots);
    size_t n_knots = 0;
    if ((st = prepare_fixed(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, h_scheme, knots_h,
                            RTB_NOALLOC_MAX_KNOTS, n_knots)) != RTB_OK)
        return st;
    const Layout l = layout(n_knots, n_beams, n_beams * ns1);
    // the packed tables move to their final offset (l.knots == l0.knots)
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
    unsigned char* d = static_cast<unsigned char*>(base);
    RTB_CUDA_TRY(cudaMemcpyAsync(d, h_stage, l.counts, cudaMemcpyHostToDevice, s));
    RTB_CUDA_TRY(cudaMemsetAsync(d + l.counts, 0, l.total - l.counts, s));

    const bool mixed = opts->precision == RTB_MIXED;
    size_t smem = fused_smem_bytes((int)n_knots);
    if (smem > (size_t)engine().max_smem_optin) return RTB_BAD_VALUE;
    auto kern = mixed ? k_fused_mixed : k_fused_fp64;
    RTB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RTB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    if (per_sm < 1) per_sm = 1;
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
    kern<<<grid_for(in->n, 256 * kDefaultRpt, per_sm), 256, smem, s>>>(
        reinterpret_cast<const DevScheme*>(d), reinterpret_cast<const double*>(d + l.knots),
        reinterpret_cast<const DevBeam*>(d + l.beams), (int)n_beams, ri, ro, counts_d, err_d,
        opts->state_out ? 1 : 0, frame, TileSched{tiles_d, kDefaultRpt});
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
