// reduce.cu -- reductions over the wavelengths of a trace's result: the
// transmission per wavelength of the reference's losses_comp
// (efficiency/losses_comp.cpp:11-136) and the distinct wavelengths of
// print_lambda (tools/print_lambda.cpp:12-90), on device arrays.
//
// Both programs sort or scan the wavelengths of every ray on the host; here
// the wavelengths are radix-sorted on the device (CUB) and only the few
// numbers of the result come back.
#include <cub/cub.cuh>

#include "engine.cuh"

namespace rtb {

namespace {

// losses_comp's counting loop (losses_comp.cpp:74-86) over the sorted
// wavelengths: ll[i] = all[i * nl]; ratio[i] = (number of good[k] == ll[i]
// for k in [cp, cp + nl)) / nl, cp advancing by that number.  The window is
// clipped to the good rays (the reference reads past them).  Sequential, as
// the loop is: one thread, a binary search per wavelength.
__global__ void k_loss_windows(const double* all, const double* good, uint64_t n_good, uint64_t n_lambda, uint64_t nl,
                               double* ll, double* ratio) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    uint64_t cp = 0;
    for (uint64_t i = 0; i < n_lambda; ++i) {
        const double v = all[i * nl];
        ll[i] = v;
        const uint64_t e = (cp + nl < n_good) ? cp + nl : n_good;
        uint64_t lo = cp, hi = e;  // first index in [cp, e) with good[k] >= v
        while (lo < hi) {
            const uint64_t m = (lo + hi) / 2;
            if (good[m] < v) lo = m + 1; else hi = m;
        }
        uint64_t a = lo, b = e;    // first index in [lo, e) with good[k] > v
        while (a < b) {
            const uint64_t m = (a + b) / 2;
            if (good[m] <= v) a = m + 1; else b = m;
        }
        // equal values are contiguous in sorted order; the reference counts
        // only those inside the window, and they start at lo
        const uint64_t cnt = a - lo;
        ratio[i] = 1.0 * (double)cnt / (double)nl;
        cp += cnt;
        if (cp > n_good) break;
    }
}

// Run heads of sorted wavelengths: the first of each run of equal values
// (NaN equals nothing, as with the reference's ==).
__global__ void k_run_heads(const double* v, uint64_t n, char* head) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x)
        head[k] = (k == 0 || !(v[k] == v[k - 1])) ? 1 : 0;
}

__global__ void k_iota(uint64_t n, unsigned long long* idx) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x)
        idx[k] = k;
}

size_t al(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

}  // namespace rtb

using namespace rtb;

extern "C" int rtb_loss_ratios(const double* lambda, uint64_t n, uint64_t n_good, uint64_t n_lambda, double* ll,
                               double* ratio, void* stream) {
    if (!lambda || !ll || !ratio || n == 0 || n_lambda == 0 || n_good > n) return RTB_BAD_VALUE;
    if (n > (uint64_t)INT32_MAX * 16) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    const uint64_t nl = n / n_lambda;
    size_t t1 = 0, t2 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, t1, (const double*)nullptr, (double*)nullptr, (int64_t)n, 0, 64, s);
    if (n_good)
        cub::DeviceRadixSort::SortKeys(nullptr, t2, (const double*)nullptr, (double*)nullptr, (int64_t)n_good, 0,
                                       64, s);
    const size_t tmp = t1 > t2 ? t1 : t2;
    const size_t o_good = al(n * 8), o_ll = o_good + al(n_good * 8 + 8), o_r = o_ll + al(n_lambda * 8),
                 o_t = o_r + al(n_lambda * 8);
    DevBuf buf;
    if ((st = buf.alloc(o_t + tmp, s)) != RTB_OK) return st;
    char* p = buf.as<char>();
    double* all = reinterpret_cast<double*>(p);
    double* good = reinterpret_cast<double*>(p + o_good);
    double* d_ll = reinterpret_cast<double*>(p + o_ll);
    double* d_r = reinterpret_cast<double*>(p + o_r);
    void* t = p + o_t;
    size_t tb = tmp;
    RTB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(t, tb, lambda, all, (int64_t)n, 0, 64, s));
    if (n_good) {
        tb = tmp;
        RTB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(t, tb, lambda, good, (int64_t)n_good, 0, 64, s));
    }
    k_loss_windows<<<1, 1, 0, s>>>(all, good, n_good, n_lambda, nl, d_ll, d_r);
    RTB_CUDA_TRY(cudaGetLastError());
    RTB_CUDA_TRY(cudaMemcpyAsync(ll, d_ll, n_lambda * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaMemcpyAsync(ratio, d_r, n_lambda * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    return RTB_OK;
}

extern "C" int rtb_unique_lambdas(const double* lambda, uint64_t n_good, uint64_t max_out, double* out,
                                  uint64_t* n_out, void* stream) {
    if (!n_out || (n_good && !lambda) || (max_out && !out)) return RTB_BAD_VALUE;
    *n_out = 0;
    if (n_good == 0 || max_out == 0) return RTB_OK;
    if (n_good > (uint64_t)INT32_MAX * 16) return RTB_BAD_VALUE;
    Lock l;
    int st = ensure_init();
    if (st != RTB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : engine().stream;
    using u64 = unsigned long long;
    const uint64_t n = n_good;
    // (value, first index) of every run of equal values, then by first index
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, (const double*)nullptr, (double*)nullptr, (const u64*)nullptr,
                                    (u64*)nullptr, (int64_t)n, 0, 64, s);
    cub::DeviceSelect::Flagged(nullptr, t2, (const double*)nullptr, (const char*)nullptr, (double*)nullptr,
                               (u64*)nullptr, (int64_t)n, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t3, (const u64*)nullptr, (u64*)nullptr, (const double*)nullptr,
                                    (double*)nullptr, (int64_t)n, 0, 64, s);
    size_t tmp = t1 > t2 ? t1 : t2;
    tmp = tmp > t3 ? tmp : t3;
    const size_t a8 = al(n * 8);
    const size_t o_idx = 0, o_sv = a8, o_si = 2 * a8, o_head = 3 * a8, o_uv = o_head + al(n), o_ui = o_uv + a8,
                 o_cnt = o_ui + a8, o_fv = o_cnt + 256, o_fi = o_fv + a8, o_t = o_fi + a8;
    DevBuf buf;
    if ((st = buf.alloc(o_t + tmp, s)) != RTB_OK) return st;
    char* p = buf.as<char>();
    u64* idx = reinterpret_cast<u64*>(p + o_idx);
    double* sv = reinterpret_cast<double*>(p + o_sv);
    u64* si = reinterpret_cast<u64*>(p + o_si);
    char* head = p + o_head;
    double* uv = reinterpret_cast<double*>(p + o_uv);
    u64* ui = reinterpret_cast<u64*>(p + o_ui);
    u64* cnt = reinterpret_cast<u64*>(p + o_cnt);
    double* fv = reinterpret_cast<double*>(p + o_fv);
    u64* fi = reinterpret_cast<u64*>(p + o_fi);
    void* t = p + o_t;
    k_iota<<<grid_for(n, 256, 8), 256, 0, s>>>(n, idx);
    size_t tb = tmp;
    // radix sort is stable: within a run the indices stay ascending, the
    // head's is the first occurrence
    RTB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tb, lambda, sv, idx, si, (int64_t)n, 0, 64, s));
    k_run_heads<<<grid_for(n, 256, 8), 256, 0, s>>>(sv, n, head);
    tb = tmp;
    RTB_CUDA_TRY(cub::DeviceSelect::Flagged(t, tb, sv, head, uv, cnt, (int64_t)n, s));
    tb = tmp;
    RTB_CUDA_TRY(cub::DeviceSelect::Flagged(t, tb, si, head, ui, cnt + 1, (int64_t)n, s));
    u64 h_cnt = 0;
    RTB_CUDA_TRY(cudaMemcpyAsync(&h_cnt, cnt, 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    tb = tmp;
    RTB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tb, ui, fi, uv, fv, (int64_t)h_cnt, 0, 64, s));
    const uint64_t m = h_cnt < max_out ? h_cnt : max_out;
    RTB_CUDA_TRY(cudaMemcpyAsync(out, fv, m * 8, cudaMemcpyDeviceToHost, s));
    RTB_CUDA_TRY(cudaStreamSynchronize(s));
    *n_out = m;
    return RTB_OK;
}
