// plan.cu -- batched traces launched as one CUDA graph, and the autotuner of
// their launch configuration.
//
// A plan fixes everything a trace of many beams needs -- prepared scheme,
// knot tables, beam table, generated rays, output arrays, loss counters and
// their page-locked host copy -- so that a run is four stream operations
// (clear the counters, the fused kernel, copy the counters back) that are
// captured once into a CUDA graph and then replayed with one
// cudaGraphLaunch.  Beams of any size, wavelength, field angle and grating
// order share the launch: the kernel finds a ray's beam from the beam table.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine.cuh"
#include "jit.h"
#include "rowpipe.cuh"

using namespace rtb;

struct rtb_plan {
    int device = 0;
    PreparedScheme ps;
    std::vector<DevBeam> beams_h;
    size_t n_beams = 0;
    uint64_t n_rays = 0;
    rtb_trace_opts opts{};
    rtb_ccd ccd{};
    bool has_frame = false;
    TraceArgs args;                  // scheme, knots, beams, counters (device)
    void* in_mem = nullptr;          // generated rays
    void* out_mem = nullptr;         // output arrays
    uint32_t* order = nullptr;       // coherent tracing order (device), or NULL for index order
    void* slot_mem = nullptr;        // the input rays in tracing order (with `order`): SoA (FP64 plans)
    DevRays in_slot{};
    void* rows = nullptr;            // or row blocks (mixed plans: Row64, Row32 for RTB_MIXED32)
    DevRays in{}, out{};
    unsigned long long* h_counts = nullptr;  // page-locked: counters, then the error word
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_stale = true;
    bool ran = false;
    int32_t block = 256, rpt = kDefaultRpt;
    uint64_t key = 0;
    std::string jit_note;            // why the generic kernel is launched ("" if specialised)
};

namespace {

// Configurations the autotuner chose, by plan key (scheme, precision, frame
// use, ray order, ray count), for the life of the process.
std::mutex g_tuned_mu;
std::map<uint64_t, std::pair<int32_t, int32_t>> g_tuned;

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

uint64_t plan_key(const rtb_plan& p) {
    uint64_t h = 1469598103934665603ull;
    h = fnv1a(h, &p.ps.sch, sizeof(DevScheme));
    h = fnv1a(h, p.ps.knots.data(), p.ps.knots.size() * sizeof(double));
    h = fnv1a(h, &p.n_rays, sizeof(p.n_rays));
    int32_t tags[5] = {p.opts.precision, p.has_frame ? 1 : 0, p.opts.ray_order, p.ps.scheme_kernel ? 1 : 0,
                       p.opts.out_order};
    return fnv1a(h, tags, sizeof(tags));
}

bool config_ok(const rtb_plan& p, int32_t block, int32_t rpt) {
    const bool mixed = p.opts.precision == RTB_MIXED || p.opts.precision == RTB_MIXED32;
    if (block != 128 && block != 256 && !(mixed && block == 512)) return false;
    return rpt >= 1 && rpt <= 64;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Carve the SoA arrays of n rays out of one block of memory.
DevRays carve(void* mem, uint64_t n, bool full) {
    char* p = static_cast<char*>(mem);
    const size_t d = align256(n * sizeof(double));
    DevRays r{};
    r.n = n;
    r.X = reinterpret_cast<double*>(p);
    r.Y = reinterpret_cast<double*>(p + d);
    size_t off = 2 * d;
    if (full) {
        r.Z = reinterpret_cast<double*>(p + off);
        r.cX = reinterpret_cast<double*>(p + off + d);
        r.cY = reinterpret_cast<double*>(p + off + 2 * d);
        r.cZ = reinterpret_cast<double*>(p + off + 3 * d);
        r.lambda = reinterpret_cast<double*>(p + off + 4 * d);
        off += 5 * d;
    }
    r.flag = reinterpret_cast<char*>(p + off);
    r.lost_stage = reinterpret_cast<uint8_t*>(p + off + align256(n));
    return r;
}

size_t rays_bytes(uint64_t n, bool full) {
    return (full ? 7 : 2) * align256(n * sizeof(double)) + 2 * align256(n);
}

// The stream operations of one run.
int enqueue_run(rtb_plan* p, const FrameArgs& frame, cudaStream_t s) {
    RTB_CUDA_TRY(cudaMemsetAsync(p->args.counts, 0, p->args.counts_len * 8, s));
    RTB_CUDA_TRY(cudaMemsetAsync(p->args.err, 0, 256, s));  // error word and tile counter
    rtb_trace_opts o = p->opts;
    o.block_size = p->block;
    o.rays_per_thread = p->rpt;
    const bool by_slot = p->opts.out_order == RTB_OUT_SLOT;
    int st = p->rows    ? launch_trace(p->ps, p->args, (int)p->n_beams, o, p->in, p->out, frame, s, p->order, true,
                                       p->rows, by_slot)
             : p->order ? launch_trace(p->ps, p->args, (int)p->n_beams, o, p->in_slot, p->out, frame, s, p->order,
                                       true, nullptr, by_slot)
                        : launch_trace(p->ps, p->args, (int)p->n_beams, o, p->in, p->out, frame, s);
    if (st != RTB_OK) return st;
    RTB_CUDA_TRY(cudaMemcpyAsync(p->h_counts, p->args.counts, p->args.counts_len * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(p->h_counts + p->args.counts_len, p->args.err, 4, cudaMemcpyDeviceToHost, s));
    return RTB_OK;
}

int capture(rtb_plan* p) {
    if (p->exec) {
        cudaGraphExecDestroy(p->exec);
        p->exec = nullptr;
    }
    FrameArgs frame = frame_args(&p->opts);
    cudaGraph_t g = nullptr;
    RTB_CUDA_TRY(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_run(p, frame, p->stream);
    cudaError_t e = cudaStreamEndCapture(p->stream, &g);
    if (st != RTB_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaGraphInstantiate(&p->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        p->exec = nullptr;
        return cuda_status(e);
    }
    p->graph_stale = false;
    return RTB_OK;
}

int run_on(rtb_plan* p, cudaStream_t s) {
    if (p->graph_stale) {
        int st = capture(p);
        if (st != RTB_OK) return st;
    }
    RTB_CUDA_TRY(cudaGraphLaunch(p->exec, s));
    RTB_CUDA_TRY(cudaEventRecord(p->done, s));
    p->ran = true;
    return RTB_OK;
}

void release(rtb_plan* p) {
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    p->args.buf.release();
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->in_mem) cudaFree(p->in_mem);
    if (p->out_mem) cudaFree(p->out_mem);
    if (p->order) cudaFree(p->order);
    if (p->slot_mem) cudaFree(p->slot_mem);
    if (p->rows) cudaFree(p->rows);
    if (p->h_counts) cudaFreeHost(p->h_counts);
    if (p->done) cudaEventDestroy(p->done);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

int rtb_plan_create(const rtb_surface* surfaces, size_t n_surfaces, const rtb_beam* beams, size_t n_beams,
                    const rtb_trace_opts* opts, rtb_plan** plan) {
    Range range("rtb_plan_create");
    if (!plan || !opts || !beams || n_beams == 0) return RTB_BAD_VALUE;
    *plan = nullptr;
    if (opts->engine != RTB_ENGINE_FUSED) return RTB_BAD_VALUE;
    if (opts->precision != RTB_FP64 && opts->precision != RTB_MIXED && opts->precision != RTB_MIXED32)
        return RTB_BAD_VALUE;
    if (opts->out_order != RTB_OUT_INDEX && opts->out_order != RTB_OUT_SLOT) return RTB_BAD_VALUE;
    // compile the kernel specialised to the scheme first, outside the engine
    // lock (NVRTC takes up to a second or so; other calls need not wait)
    if (specialize_enabled()) {
        PreparedScheme pre;
        if (prepare_scheme(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, pre) == RTB_OK)
            compile_scheme(pre.sch, opts->precision, nullptr);
    }
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    rtb_plan* p = new rtb_plan();
    cudaGetDevice(&p->device);
    p->opts = *opts;
    p->has_frame = opts->ccd && opts->counts;
    if (p->has_frame) {
        p->ccd = *opts->ccd;
        p->opts.ccd = &p->ccd;
        if (p->ccd.xdim == 0 || p->ccd.ydim == 0) {
            delete p;
            return RTB_BAD_VALUE;
        }
    } else {
        p->opts.ccd = nullptr;
        p->opts.counts = nullptr;
        p->opts.n_outside = nullptr;
    }
    p->n_beams = n_beams;
    p->n_rays = beams[n_beams - 1].first_ray + beams[n_beams - 1].n_rays;
    std::vector<GenBeam> gb;
    uint64_t total = 0;
    if ((st = prepare_scheme(surfaces, n_surfaces, opts->fixes, opts->renormalize_lost, p->ps)) != RTB_OK ||
        (st = check_beams(beams, n_beams, p->n_rays, p->beams_h, &p->ps.sch)) != RTB_OK ||
        (st = gen_beams(beams, n_beams, p->n_rays, gb, &total)) != RTB_OK) {
        delete p;
        return st;
    }
    if (!specialize_enabled()) {
        p->jit_note = "RTB_SPECIALIZE=0";
    } else if ((st = scheme_kernel(p->ps.sch, opts->precision, &p->ps.scheme_kernel, &p->jit_note)) != RTB_OK) {
        delete p;
        return st;
    }
    if (opts->block_size > 0 || opts->rays_per_thread > 0) {
        p->block = opts->block_size > 0 ? opts->block_size : 256;
        p->rpt = opts->rays_per_thread > 0 ? opts->rays_per_thread : kDefaultRpt;
        if (!config_ok(*p, p->block, p->rpt)) {
            delete p;
            return RTB_BAD_VALUE;
        }
    }
    p->key = plan_key(*p);
    if (opts->block_size <= 0 && opts->rays_per_thread <= 0) {
        std::lock_guard<std::mutex> g(g_tuned_mu);
        auto it = g_tuned.find(p->key);
        if (it != g_tuned.end()) {
            p->block = it->second.first;
            p->rpt = it->second.second;
        }
    }
    const bool full_out = opts->state_out != 0;
    cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = dev_malloc((void**)&p->in_mem, rays_bytes(p->n_rays, true));
    if (e == cudaSuccess) e = dev_malloc((void**)&p->out_mem, rays_bytes(p->n_rays, full_out));
    if (e == cudaSuccess)
        e = cudaMallocHost(&p->h_counts, (n_beams * (3 * n_surfaces + 1) + 1) * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        release(p);
        return cuda_status(e);
    }
    p->in = carve(p->in_mem, p->n_rays, true);
    p->out = carve(p->out_mem, p->n_rays, full_out);
    p->out.lambda = p->in.lambda;
    if ((st = p->args.init(p->ps, p->beams_h, p->stream)) != RTB_OK) {
        release(p);
        return st;
    }
    // generate the rays once
    DevBuf gbuf;
    if ((st = gbuf.alloc(n_beams * sizeof(GenBeam), p->stream)) != RTB_OK) {
        release(p);
        return st;
    }
    e = cudaMemcpyAsync(gbuf.p, gb.data(), n_beams * sizeof(GenBeam), cudaMemcpyHostToDevice, p->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->in.flag, 0, p->n_rays, p->stream);  // rays outside every beam
    if (e == cudaSuccess) {
        k_generate<<<grid_for(total, 256, 8), 256, 0, p->stream>>>(gbuf.as<GenBeam>(), (int)n_beams, total, p->in);
        e = cudaGetLastError();
    }
    // the coherent tracing order and a copy of the rays in that order, once
    // (index order for plans beyond 2^32 rays).  The rays of a beam are
    // grouped by wavelength within chunks of 2^20 consecutive rays for the
    // mixed kernel and of the whole beam (up to 2^30) for the FP64 kernel:
    // the best of 2^11..2^30 for each on C1 (mixed: 5.24 ms at 2^20, 5.36
    // whole beams, 5.65 at 2^11; FP64: 24.7 ms whole beams, 25.1 at 2^20).
    // Outputs are stored at the rays' indices, 8 bytes apart per lane, which
    // costs the mixed kernel 0.8 ms of its 5.3 on C1 against coalesced stores;
    // chunks small enough to stage a block's stores in shared memory lose
    // more in coherence than that.
    // The order is beam-major (k_order_keys): the slots of beam b are the
    // range of its ray indices, so a kernel reading rows finds a ray's beam
    // from its slot.  The mixed kernels read the ordered copy as row blocks of 32 rays
    // (rowpipe.cuh: one bulk copy per row into shared memory, issued a row
    // ahead), the FP32-state kernel with FP32 positions relative to each
    // beam's origin: 57 and 33 bytes per ray.
    const bool mixed = opts->precision != RTB_FP64;
    if (e == cudaSuccess && opts->ray_order == RTB_ORDER_COHERENT && p->n_rays <= 0xffffffffull) {
        e = dev_malloc((void**)&p->order, p->n_rays * sizeof(uint32_t));
        const size_t n_rows = (p->n_rays + 31) / 32;
        const size_t row_size = opts->precision == RTB_MIXED32 ? sizeof(Row32) : sizeof(Row64);
        if (e == cudaSuccess)
            e = mixed ? dev_malloc((void**)&p->rows, n_rows * row_size) : dev_malloc((void**)&p->slot_mem, rays_bytes(p->n_rays, true));
        if (e == cudaSuccess) {
            if (!mixed) p->in_slot = carve(p->slot_mem, p->n_rays, true);
            const int chunk_shift = mixed ? 20 : 30;
            st = coherent_order(gbuf.as<GenBeam>(), (int)n_beams, p->n_rays, p->in, p->order, chunk_shift,
                                p->stream);
            if (st == RTB_OK) {
                const unsigned g = grid_for(n_rows * 32, 256, 8);
                if (opts->precision == RTB_MIXED32)
                    k_gather_rows32<<<g, 256, 0, p->stream>>>(p->order, p->n_rays, p->in, p->args.beams,
                                                              (int)n_beams, p->rows);
                else if (mixed)
                    k_gather_rows64<<<g, 256, 0, p->stream>>>(p->order, p->n_rays, p->in, p->rows);
                else
                    k_gather_rays<<<grid_for(p->n_rays, 256, 8), 256, 0, p->stream>>>(p->order, p->n_rays, p->in,
                                                                                      p->in_slot);
                e = cudaGetLastError();
            }
            if (st != RTB_OK) {
                gbuf.release();
                release(p);
                return st;
            }
        }
    } else if (e == cudaSuccess && opts->ray_order != RTB_ORDER_COHERENT && opts->ray_order != RTB_ORDER_INDEX) {
        gbuf.release();
        release(p);
        return RTB_BAD_VALUE;
    }
    gbuf.release();
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) {
        release(p);
        return cuda_status(e);
    }
    *plan = p;
    return RTB_OK;
}

int rtb_plan_run(rtb_plan* p, void* stream) {
    Range range("rtb_plan_run");
    if (!p) return RTB_BAD_VALUE;
    DeviceGuard dg(p->device);
    Lock l;
    return run_on(p, stream ? (cudaStream_t)stream : p->stream);
}

int rtb_plan_result(rtb_plan* p, rtb_trace_stats* stats) {
    if (!p || !p->ran) return RTB_BAD_VALUE;
    DeviceGuard dg(p->device);
    RTB_CUDA_TRY(cudaEventSynchronize(p->done));
    unsigned err = (unsigned)(p->h_counts[p->args.counts_len] & 0xffffffffu);
    return trace_result(p->ps, p->h_counts, err, (int)p->n_beams, stats);
}

int rtb_plan_counts(rtb_plan* p, uint64_t* counts, size_t capacity, size_t* n_entries) {
    if (!p || !p->ran) return RTB_BAD_VALUE;
    DeviceGuard dg(p->device);
    RTB_CUDA_TRY(cudaEventSynchronize(p->done));
    const size_t n = p->args.counts_len;
    if (n_entries) *n_entries = n;
    if (counts) std::memcpy(counts, p->h_counts, (capacity < n ? capacity : n) * sizeof(uint64_t));
    return RTB_OK;
}

int rtb_plan_order(const rtb_plan* p, const uint32_t** order) {
    if (!p || !order) return RTB_BAD_VALUE;
    *order = p->order;
    return RTB_OK;
}

int rtb_plan_rays(const rtb_plan* p, rtb_rays* in, rtb_rays* out) {
    if (!p) return RTB_BAD_VALUE;
    auto put = [](const DevRays& d, rtb_rays* r) {
        r->X = d.X; r->Y = d.Y; r->Z = d.Z; r->cX = d.cX; r->cY = d.cY; r->cZ = d.cZ;
        r->lambda = d.lambda;
        r->flag = d.flag;
        r->lost_stage = d.lost_stage;
        r->n = d.n;
    };
    if (in) put(p->in, in);
    if (out) put(p->out, out);
    return RTB_OK;
}

int rtb_plan_set_config(rtb_plan* p, int32_t block, int32_t rpt) {
    if (!p || !config_ok(*p, block, rpt)) return RTB_BAD_VALUE;
    if (block != p->block || rpt != p->rpt) {
        p->block = block;
        p->rpt = rpt;
        p->graph_stale = true;
    }
    return RTB_OK;
}

int rtb_plan_config(const rtb_plan* p, int32_t* block, int32_t* rpt, uint64_t* n_rays) {
    if (!p) return RTB_BAD_VALUE;
    if (block) *block = p->block;
    if (rpt) *rpt = p->rpt;
    if (n_rays) *n_rays = p->n_rays;
    return RTB_OK;
}

int rtb_plan_autotune(rtb_plan* p, int reps, rtb_tune_entry* table, size_t capacity, size_t* n_entries) {
    Range range("rtb_plan_autotune");
    if (!p || reps < 1) return RTB_BAD_VALUE;
    DeviceGuard dg(p->device);
    Lock l;
    const int32_t blocks[3] = {128, 256, 512};
    const int32_t rpts[4] = {1, 2, 4, 8};
    // the sweep writes to a private frame, so the caller's stays untouched
    const rtb_trace_opts saved = p->opts;
    const int32_t saved_block = p->block, saved_rpt = p->rpt;
    void* frame_mem = nullptr;
    if (p->has_frame) {
        RTB_CUDA_TRY(dev_malloc((void**)&frame_mem, p->ccd.xdim * p->ccd.ydim * sizeof(uint32_t) + 256));
        p->opts.counts = static_cast<uint32_t*>(frame_mem);
        p->opts.n_outside = reinterpret_cast<uint64_t*>(static_cast<char*>(frame_mem) +
                                                        p->ccd.xdim * p->ccd.ydim * sizeof(uint32_t));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = RTB_OK;
    double best_ms = 1e300;
    int32_t best_b = saved_block, best_r = saved_rpt;
    size_t n = 0;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = RTB_FAILED;
    for (int bi = 0; bi < 3 && st == RTB_OK; ++bi) {
        for (int ri = 0; ri < 4 && st == RTB_OK; ++ri) {
            if (!config_ok(*p, blocks[bi], rpts[ri])) continue;
            p->block = blocks[bi];
            p->rpt = rpts[ri];
            p->graph_stale = true;
            if ((st = run_on(p, p->stream)) != RTB_OK) break;  // untimed: capture and warm-up
            if (cudaEventRecord(e0, p->stream) != cudaSuccess) { st = RTB_FAILED; break; }
            for (int k = 0; k < reps && st == RTB_OK; ++k) st = run_on(p, p->stream);
            if (st != RTB_OK) break;
            float ms = 0.f;
            if (cudaEventRecord(e1, p->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                st = RTB_FAILED;
                break;
            }
            const double per = (double)ms / reps;
            if (table && n < capacity) table[n] = rtb_tune_entry{p->block, p->rpt, per};
            ++n;
            if (per < best_ms) {
                best_ms = per;
                best_b = p->block;
                best_r = p->rpt;
            }
        }
    }
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (frame_mem) cudaFree(frame_mem);
    p->opts = saved;
    p->block = (st == RTB_OK) ? best_b : saved_block;
    p->rpt = (st == RTB_OK) ? best_r : saved_rpt;
    p->graph_stale = true;
    p->ran = false;  // the counters of the sweep are not a result of the plan's own configuration
    if (n_entries) *n_entries = n;
    if (st == RTB_OK) {
        std::lock_guard<std::mutex> g(g_tuned_mu);
        g_tuned[p->key] = {best_b, best_r};
    }
    return st;
}

int rtb_plan_specialized(const rtb_plan* p, int32_t* specialized, char* note, size_t note_len) {
    if (!p || !specialized) return RTB_BAD_VALUE;
    *specialized = p->ps.scheme_kernel ? 1 : 0;
    if (note && note_len > 0) std::snprintf(note, note_len, "%s", p->jit_note.c_str());
    return RTB_OK;
}

int rtb_plan_destroy(rtb_plan* p) {
    if (!p) return RTB_OK;
    DeviceGuard dg(p->device);
    release(p);
    return RTB_OK;
}

}  // extern "C"
