// engine.cuh -- host-side state and helpers of the C ABI.
#pragma once

#include <mutex>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kernels.cuh"

namespace rtb {

struct Engine {
    std::mutex mu;
    bool inited = false;
    int device = 0;
    int sm_count = 148;
    int max_smem_optin = 0;
    cudaStream_t stream = nullptr;
};

Engine& engine();
int ensure_init();

// Fault hook (rtb_fail_allocations): true for the allocations it makes fail.
bool injected_alloc_failure();
// cudaMalloc, failing as out of memory while the fault hook says so.
cudaError_t dev_malloc(void** p, size_t bytes);

// Host-side scheme preparation (what the reference's host code computes
// before its launches).
struct PreparedScheme {
    DevScheme sch;
    std::vector<double> knots;
    // fused traces launch this kernel (a copy of k_fused_mixed or
    // k_fused_fp64, of the trace's precision, specialised to the scheme;
    // jit.cpp) instead of the generic one when set
    const void* scheme_kernel = nullptr;
};

// The knot buffer a scheme's tables are packed into: a growing vector, or a
// fixed array of `cap` doubles (the no-allocation trace), which refuses what
// does not fit.
struct KnotBuf {
    std::vector<double>* vec = nullptr;
    double* fixed = nullptr;
    size_t cap = 0, n = 0;
    explicit KnotBuf(std::vector<double>& v) : vec(&v) {}
    KnotBuf(double* p, size_t capacity) : fixed(p), cap(capacity) {}
    bool append(const double* v, size_t k);
    size_t size() const { return vec ? vec->size() : n; }
    const double* data() const { return vec ? vec->data() : fixed; }
};

int prepare_surface(const rtb_surface& in, DevSurface& out, KnotBuf& knots);
// Every launch of a scheme reads what this prepares: the surfaces' constants,
// the packed tables (identical tables sharing one copy, the inverse spacing
// of tables on a uniform grid) and the counts that follow from the sequence.
int prepare_scheme_into(const rtb_surface* s, size_t n, uint32_t fixes, int renorm_lost, DevScheme& sch,
                        KnotBuf& knots);
int prepare_scheme(const rtb_surface* s, size_t n, uint32_t fixes, int renorm_lost, PreparedScheme& out);
int surface_from_params(int cls, const double* params, DevSurface& s);
int add_table(const rtb_table* t, KnotBuf& knots, int32_t& off, int32_t& cnt);
int add_table(const rtb_table* t, std::vector<double>& knots, int32_t& off, int32_t& cnt);
// Sag range of an even asphere over its circular aperture (DevSurface::sag_*).
void asphere_sag_bounds(DevSurface& s);
// The mixed engine's per-surface constants: the sag range and inv_c, inv_gr.
void mixed_constants(DevSurface& s);
void transform_constants(const double angles_rad[3], const double dist[3], DevSurface& s);
double scheme_angle_rad(double deg);

// Grid for a grid-stride kernel over n items.
inline unsigned grid_for(size_t n, int threads, int per_sm) {
    size_t blocks = (n + threads - 1) / threads;
    size_t cap = (size_t)engine().sm_count * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    return (unsigned)blocks;
}

// A device allocation released at scope exit (stream-ordered).
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
    }
    int alloc(size_t bytes, cudaStream_t st) {
        release();
        s = st;
        cudaError_t e = injected_alloc_failure() ? cudaErrorMemoryAllocation
                                                 : cudaMallocAsync(&p, bytes ? bytes : 16, st);
        if (e != cudaSuccess) {
            p = nullptr;
            return cuda_status(e);
        }
        return RTB_OK;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// ---- trace plumbing shared by the C ABI files (trace.cu) ----

struct Lock {
    std::lock_guard<std::mutex> g;
    Lock() : g(engine().mu) {}
};

// A named range of a C ABI call on a profiler's timeline (NVTX, domain
// "rt_b200"), from construction to destruction; a no-op when no tool is
// attached.  Kernels and copies the call enqueues show under it.
struct Range {
    nvtxDomainHandle_t dom;
    explicit Range(const char* name) {
        static nvtxDomainHandle_t d = nvtxDomainCreateA("rt_b200");
        dom = d;
        nvtxEventAttributes_t a = {};
        a.version = NVTX_VERSION;
        a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
        a.messageType = NVTX_MESSAGE_TYPE_ASCII;
        a.message.ascii = name;
        nvtxDomainRangePushEx(dom, &a);
    }
    ~Range() { nvtxDomainRangePop(dom); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Everything a trace launch reads, in one pool allocation.
struct TraceArgs {
    DevBuf buf;
    DevScheme* sch;
    double* knots;
    DevBeam* beams;
    unsigned long long* counts;
    unsigned* err;
    unsigned long long* tiles;  // tile counter of the fused kernels
    size_t counts_len;
    int init(const PreparedScheme& ps, const std::vector<DevBeam>& beams_h, cudaStream_t st) {
        size_t n_beams = beams_h.size();
        counts_len = n_beams * (size_t)(3 * ps.sch.n_surfaces + 1);
        size_t off_knots = (sizeof(DevScheme) + 255) / 256 * 256;
        size_t off_beams = off_knots + (ps.knots.size() * sizeof(double) + 255) / 256 * 256;
        size_t off_counts = off_beams + (n_beams * sizeof(DevBeam) + 255) / 256 * 256;
        size_t off_err = off_counts + (counts_len * 8 + 255) / 256 * 256;
        int s = buf.alloc(off_err + 256, st);
        if (s != RTB_OK) return s;
        char* p = buf.as<char>();
        sch = reinterpret_cast<DevScheme*>(p);
        knots = reinterpret_cast<double*>(p + off_knots);
        beams = reinterpret_cast<DevBeam*>(p + off_beams);
        counts = reinterpret_cast<unsigned long long*>(p + off_counts);
        err = reinterpret_cast<unsigned*>(p + off_err);
        tiles = reinterpret_cast<unsigned long long*>(p + off_err + 64);
        RTB_CUDA_TRY(cudaMemcpyAsync(sch, &ps.sch, sizeof(DevScheme), cudaMemcpyHostToDevice, st));
        RTB_CUDA_TRY(cudaMemcpyAsync(knots, ps.knots.data(), ps.knots.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        RTB_CUDA_TRY(cudaMemcpyAsync(beams, beams_h.data(), n_beams * sizeof(DevBeam), cudaMemcpyHostToDevice, st));
        RTB_CUDA_TRY(cudaMemsetAsync(counts, 0, counts_len * 8, st));
        RTB_CUDA_TRY(cudaMemsetAsync(err, 0, 256, st));  // err and the tile counter
        return RTB_OK;
    }
};

DevRays dev_rays(const rtb_rays* r);
// Beam table for the trace kernels; rays of beam b are [first_ray, first_ray + n_rays) < n_rays, in order.
// With `sch`, each beam also gets its origin and first-surface offset for the
// FP32-state engine (beam_frame).
int check_beams(const rtb_beam* beams, size_t n_beams, size_t n_rays, std::vector<DevBeam>& out,
                const DevScheme* sch = nullptr);
// A beam's origin (its centre: FP32 positions are relative to it) and the
// offset of the first non-Aux surface's transform for such positions.
void beam_frame(const DevScheme& sch, const double center[3], DevBeam& d);
// Beam table for the generator; *total is the end of the last beam.
int gen_beams(const rtb_beam* beams, size_t n_beams, size_t n_rays, std::vector<GenBeam>& out, uint64_t* total);
FrameArgs frame_args(const rtb_trace_opts* o);
// Launch the trace kernels of one call (no synchronisation).
// `order` (fused kernels; may be NULL): the order in which the rays are
// traced; in_by_slot: `in` holds the rays in that order.
// `rows` (mixed kernels; may be NULL): the rays in tracing order as row
// blocks (Row64 / Row32 of rowpipe.cuh), read in place of `in`;
// out_by_slot: outputs at the tracing slot instead of the ray's index.
int launch_trace(const PreparedScheme& ps, TraceArgs& a, int n_beams, const rtb_trace_opts& o, const DevRays& in,
                 const DevRays& out, const FrameArgs& frame, cudaStream_t st, const uint32_t* order = nullptr,
                 bool in_by_slot = false, const void* rows = nullptr, bool out_by_slot = false);
// The coherent tracing order (beam, chunk, wavelength, Morton code of the
// entrance position) of n <= 2^32 generated rays, as a permutation in
// `order` (device, n).
int coherent_order(const GenBeam* d_beams, int n_beams, uint64_t n, const DevRays& rays, uint32_t* order,
                   int chunk_shift, cudaStream_t st);
// Status and statistics from the per-(beam, stage) counts.
int trace_result(const PreparedScheme& ps, const unsigned long long* counts, unsigned err, int n_beams,
                 rtb_trace_stats* stats);

}  // namespace rtb
