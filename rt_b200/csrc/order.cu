// order.cu -- the reference's Rearrange on the device.
//
// Beam::Rearrange (common-lib/beam.cpp:574-598) partitions the good prefix
// [0, ng) with two pointers: scanning from the front for lost rays and from
// the back for good rays, it swaps each pair.  The k-th lost ray in [0, N')
// (N' = ng - lost) therefore trades places with the k-th good ray of
// [N', ng) counted from the back; every other ray stays.  Here that pairing
// is computed in parallel from a prefix sum of the lost marks.
//
// reference_order() replays the Rearrange calls of a whole trace from the
// per-ray lost stages (one partition per stage with losses, all beams at
// once), giving the order in which the reference's Beam::Save writes rays.
#include <cub/cub.cuh>

#include "engine.cuh"
#include "mixed32.cuh"
#include "rowpipe.cuh"

namespace rtb {

namespace {

// Segment s covers positions [start, start + ng) of the order array.
struct Seg {
    uint64_t start, ng;
};

__device__ __forceinline__ int seg_of(const Seg* segs, int n_segs, uint64_t k) {
    int lo = 0, hi = n_segs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (segs[mid].start <= k) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_mark_stage(uint64_t n, const Seg* segs, int n_segs, const uint32_t* order, const uint8_t* lost_stage,
                             int stage, uint32_t* mark) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x) {
        int s = seg_of(segs, n_segs, k);
        bool in = k < segs[s].start + segs[s].ng;
        mark[k] = (in && lost_stage[segs[s].start + order[k]] == stage) ? 1u : 0u;
    }
}

// Per segment: lost count = rank[start+ng] - rank[start].
__global__ void k_seg_counts(const Seg* segs, int n_segs, const uint32_t* rank, const uint32_t* mark,
                             uint64_t* seg_lost) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_segs) return;
    uint64_t a = segs[s].start, b = segs[s].start + segs[s].ng;
    uint64_t ra = rank[a];
    uint64_t rb = (segs[s].ng > 0) ? (uint64_t)rank[b - 1] + mark[b - 1] : ra;
    seg_lost[s] = rb - ra;
}

// Good rays at the back of each segment record their rank from the back.
__global__ void k_back_slots(uint64_t n, const Seg* segs, int n_segs, const uint32_t* mark, const uint32_t* rank,
                             const uint64_t* seg_lost, uint64_t* slot_pos) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x) {
        int s = seg_of(segs, n_segs, k);
        uint64_t start = segs[s].start, ng = segs[s].ng, lost = seg_lost[s];
        if (lost == 0 || k >= start + ng) continue;
        uint64_t np = ng - lost;  // N'
        uint64_t j = k - start;
        if (j < np || mark[k]) continue;
        uint64_t lost_before = rank[k] - rank[start];
        uint64_t lost_after = lost - lost_before;                  // mark[k] == 0
        uint64_t good_after = (ng - 1 - j) - lost_after;
        slot_pos[start + good_after] = k;                           // rank from the back
    }
}

// Lost rays at the front swap with their partner.
template <class SwapFn>
__device__ __forceinline__ void pair_front(uint64_t k, const Seg* segs, int n_segs, const uint32_t* mark,
                                           const uint32_t* rank, const uint64_t* seg_lost, const uint64_t* slot_pos,
                                           SwapFn swap) {
    int s = seg_of(segs, n_segs, k);
    uint64_t start = segs[s].start, ng = segs[s].ng, lost = seg_lost[s];
    if (lost == 0 || k >= start + ng || !mark[k]) return;
    uint64_t np = ng - lost;
    if (k - start >= np) return;
    uint64_t r = rank[k] - rank[start];
    swap(k, slot_pos[start + r]);
}

__global__ void k_swap_order(uint64_t n, const Seg* segs, int n_segs, const uint32_t* mark, const uint32_t* rank,
                             const uint64_t* seg_lost, const uint64_t* slot_pos, uint32_t* order) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x)
        pair_front(k, segs, n_segs, mark, rank, seg_lost, slot_pos, [&](uint64_t a, uint64_t b) {
            uint32_t t = order[a];
            order[a] = order[b];
            order[b] = t;
        });
}

struct Arr7 {
    double* a[7];
};

__global__ void k_swap_arrays(uint64_t n, const Seg* segs, const uint32_t* mark, const uint32_t* rank,
                              const uint64_t* seg_lost, const uint64_t* slot_pos, Arr7 arr, char* flag) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x)
        pair_front(k, segs, 1, mark, rank, seg_lost, slot_pos, [&](uint64_t a, uint64_t b) {
            for (int i = 0; i < 7; ++i) {
                double t = arr.a[i][a];
                arr.a[i][a] = arr.a[i][b];
                arr.a[i][b] = t;
            }
            flag[a] = 1;
            flag[b] = 0;
        });
}

__global__ void k_seg_update(Seg* segs, int n_segs, const uint64_t* seg_lost) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n_segs) segs[s].ng -= seg_lost[s];
}

__global__ void k_iota(uint64_t n, const Seg* segs, int n_segs, uint32_t* order) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)blockDim.x * gridDim.x) {
        int s = seg_of(segs, n_segs, k);
        order[k] = (uint32_t)(k - segs[s].start);
    }
}

__global__ void k_mark_flags(uint64_t ng, const char* flag, uint32_t* mark) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < ng; k += (uint64_t)blockDim.x * gridDim.x)
        mark[k] = flag[k] == 0 ? 1u : 0u;
}

// Workspace: mark, rank (uint32) and slot positions (uint64) over n positions.
struct Work {
    DevBuf buf, scan;
    uint32_t *mark, *rank;
    uint64_t *slot, *seg_lost;
    Seg* segs;
    size_t scan_bytes = 0;
    int init(uint64_t n, int n_segs, cudaStream_t st) {
        size_t bytes = n * 8 + n * 8 + 64 + n_segs * (sizeof(Seg) + 8) + 64;
        int s = buf.alloc(bytes, st);
        if (s != RTB_OK) return s;
        char* p = buf.as<char>();
        slot = reinterpret_cast<uint64_t*>(p);
        p += n * 8;
        mark = reinterpret_cast<uint32_t*>(p);
        p += n * 4;
        rank = reinterpret_cast<uint32_t*>(p);
        p += n * 4 + 64;
        segs = reinterpret_cast<Seg*>(p);
        p += n_segs * sizeof(Seg);
        seg_lost = reinterpret_cast<uint64_t*>(p);
        cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, mark, rank, (int64_t)n, st);
        return scan.alloc(scan_bytes, st);
    }
    int exclusive_scan(uint64_t n, cudaStream_t st) {
        RTB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(scan.p, scan_bytes, mark, rank, (int64_t)n, st));
        return RTB_OK;
    }
};

}  // namespace

int reference_order(const DevBeam* h_beams, int n_beams, int n_stages, const DevRays& rays, uint32_t* order,
                    cudaStream_t st) {
    uint64_t n = rays.n;
    if (n == 0) return RTB_OK;
    if (n > 0xFFFFFFFFull) return RTB_BAD_VALUE;
    std::vector<Seg> segs(n_beams);
    for (int b = 0; b < n_beams; ++b) {
        segs[b].start = h_beams[b].first_ray;
        segs[b].ng = h_beams[b].n_rays;
        if (b > 0 && segs[b].start < segs[b - 1].start + segs[b - 1].ng) return RTB_BAD_VALUE;
    }
    Work w;
    int s = w.init(n, n_beams, st);
    if (s != RTB_OK) return s;
    RTB_CUDA_TRY(cudaMemcpyAsync(w.segs, segs.data(), n_beams * sizeof(Seg), cudaMemcpyHostToDevice, st));
    unsigned grid = grid_for(n, 256, 8);
    unsigned sg = (unsigned)((n_beams + 255) / 256);
    k_iota<<<grid, 256, 0, st>>>(n, w.segs, n_beams, order);
    for (int stage = 0; stage < n_stages; ++stage) {
        k_mark_stage<<<grid, 256, 0, st>>>(n, w.segs, n_beams, order, rays.lost_stage, stage, w.mark);
        if ((s = w.exclusive_scan(n, st)) != RTB_OK) return s;
        k_seg_counts<<<sg, 256, 0, st>>>(w.segs, n_beams, w.rank, w.mark, w.seg_lost);
        k_back_slots<<<grid, 256, 0, st>>>(n, w.segs, n_beams, w.mark, w.rank, w.seg_lost, w.slot);
        k_swap_order<<<grid, 256, 0, st>>>(n, w.segs, n_beams, w.mark, w.rank, w.seg_lost, w.slot, order);
        k_seg_update<<<sg, 256, 0, st>>>(w.segs, n_beams, w.seg_lost);
    }
    RTB_CUDA_TRY(cudaGetLastError());
    return RTB_OK;
}

int rearrange_device(size_t ng, double* arrays[7], char* flag, size_t* ng_out, cudaStream_t st) {
    if (ng == 0) {
        *ng_out = 0;
        return RTB_OK;
    }
    Work w;
    int s = w.init(ng, 1, st);
    if (s != RTB_OK) return s;
    Seg seg{0, ng};
    RTB_CUDA_TRY(cudaMemcpyAsync(w.segs, &seg, sizeof(Seg), cudaMemcpyHostToDevice, st));
    unsigned grid = grid_for(ng, 256, 8);
    k_mark_flags<<<grid, 256, 0, st>>>(ng, flag, w.mark);
    if ((s = w.exclusive_scan(ng, st)) != RTB_OK) return s;
    k_seg_counts<<<1, 32, 0, st>>>(w.segs, 1, w.rank, w.mark, w.seg_lost);
    k_back_slots<<<grid, 256, 0, st>>>(ng, w.segs, 1, w.mark, w.rank, w.seg_lost, w.slot);
    Arr7 arr;
    for (int i = 0; i < 7; ++i) arr.a[i] = arrays[i];
    k_swap_arrays<<<grid, 256, 0, st>>>(ng, w.segs, w.mark, w.rank, w.seg_lost, w.slot, arr, flag);
    uint64_t lost = 0;
    RTB_CUDA_TRY(cudaMemcpyAsync(&lost, w.seg_lost, sizeof(lost), cudaMemcpyDeviceToHost, st));
    RTB_CUDA_TRY(cudaStreamSynchronize(st));
    *ng_out = ng - lost;
    return RTB_OK;
}

// ---------------------------------------------------------------------------
// Coherent tracing order of generated rays.  A composite beam interleaves its
// wavelengths (ray j has wavelength j mod n_lambda) and draws positions
// independently, so the 32 rays of a warp go to 32 wavelengths and 32 points
// of the pupil, and which surface loses each of them is close to random: the
// lanes of rays lost early idle while the others finish the scheme.  Sorted
// by (beam, chunk of 2^chunk_shift consecutive rays, wavelength, Morton code
// of the entrance position), a warp traces neighbouring rays of one
// wavelength, which mostly share their fate.  The key only orders the work:
// any key gives a permutation.

__device__ __forceinline__ uint32_t spread12(uint32_t v) {
    v &= 0xfffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__global__ void k_order_keys(const GenBeam* beams, int n_beams, uint64_t total, DevRays rays,
                             unsigned long long* keys, uint32_t* idx, int chunk_shift) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)blockDim.x * gridDim.x) {
        int lo = 0, hi = n_beams - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (beams[mid].first_ray <= i) lo = mid; else hi = mid - 1;
        }
        const GenBeam& b = beams[lo];
        const uint64_t j = i - b.first_ray;
        const uint64_t lam = (j < b.n_rays && b.n_lambda > 0) ? j % b.n_lambda : 0;
        const double R = b.disk[2] > 0 ? b.disk[2] : 1.0;
        auto q = [R](double v, double c) {
            double u = (v - c) / (2.0 * R) + 0.5;
            u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
            return (uint32_t)(u * 4095.0);
        };
        const uint32_t m = spread12(q(rays.X[i], b.center[0])) | (spread12(q(rays.Y[i], b.center[1])) << 1);
        const uint64_t chunk = j >> chunk_shift;
        keys[i] = ((unsigned long long)(lo & 0xffff) << 48) | ((unsigned long long)(chunk & 0xfffu) << 36) |
                  ((unsigned long long)(lam & 0xfffu) << 24) | m;
        idx[i] = (uint32_t)i;
    }
}

int coherent_order(const GenBeam* d_beams, int n_beams, uint64_t n, const DevRays& rays, uint32_t* order,
                   int chunk_shift, cudaStream_t st) {
    if (n == 0) return RTB_OK;
    if (n > 0xffffffffull) return RTB_BAD_VALUE;
    DevBuf buf;
    const size_t kb = (n * 8 + 255) / 256 * 256, ib = (n * 4 + 255) / 256 * 256;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                    (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)n, 0, 64, st);
    int s = buf.alloc(2 * kb + ib + tmp + 256, st);
    if (s != RTB_OK) return s;
    char* p = buf.as<char>();
    auto* k_in = reinterpret_cast<unsigned long long*>(p);
    auto* k_out = reinterpret_cast<unsigned long long*>(p + kb);
    auto* i_in = reinterpret_cast<uint32_t*>(p + 2 * kb);
    void* t = p + 2 * kb + ib;
    k_order_keys<<<grid_for(n, 256, 8), 256, 0, st>>>(d_beams, n_beams, n, rays, k_in, i_in, chunk_shift);
    RTB_CUDA_TRY(cudaGetLastError());
    RTB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(t, tmp, k_in, k_out, i_in, order, (int64_t)n, 0, 64, st));
    return RTB_OK;
}

__global__ void k_gather_rays(const uint32_t* order, uint64_t n, DevRays src, DevRays dst) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)blockDim.x * gridDim.x) {
        const uint64_t i = order[t];
        dst.X[t] = src.X[i];
        dst.Y[t] = src.Y[i];
        dst.Z[t] = src.Z[i];
        dst.cX[t] = src.cX[i];
        dst.cY[t] = src.cY[i];
        dst.cZ[t] = src.cZ[i];
        dst.lambda[t] = src.lambda[i];
        dst.flag[t] = src.flag[i];
    }
}

// Row blocks of the tracing order (rowpipe.cuh): slot t goes to element
// t % 32 of row t / 32; the slots after the last ray, up to a whole row, get
// flag 0.  Each thread writes one slot, so a warp writes 32 consecutive
// elements of each component.
__global__ void k_gather_rows64(const uint32_t* order, uint64_t n, DevRays src, void* rows) {
    Row64* dst = static_cast<Row64*>(rows);
    const uint64_t total = (n + 31) / 32 * 32;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)blockDim.x * gridDim.x) {
        Row64& w = dst[t >> 5];
        const int l = (int)(t & 31);
        if (t < n) {
            const uint64_t i = order ? order[t] : t;
            // the cosines normalised as the kernel would on load (mx::normalize)
            mx::Ray r{src.X[i], src.Y[i], src.Z[i], src.cX[i], src.cY[i], src.cZ[i]};
            mx::normalize(r);
            w.X[l] = r.X;
            w.Y[l] = r.Y;
            w.Z[l] = r.Z;
            w.cX[l] = r.cX;
            w.cY[l] = r.cY;
            w.cZ[l] = r.cZ;
            w.lambda[l] = src.lambda[i];
            w.flag[l] = src.flag[i];
        } else {
            w.X[l] = w.Y[l] = w.Z[l] = w.cX[l] = w.cY[l] = w.cZ[l] = w.lambda[l] = 0.0;
            w.flag[l] = 0;
        }
    }
}

// The same with FP32 positions relative to the ray's beam's origin
// (DevBeam::origin) and FP32 cosines; the wavelength stays FP64.  Both
// gathers store the cosines normalised, so the kernels skip that on rows.
__global__ void k_gather_rows32(const uint32_t* order, uint64_t n, DevRays src, const DevBeam* beams, int n_beams,
                                void* rows) {
    Row32* dst = static_cast<Row32*>(rows);
    const uint64_t total = (n + 31) / 32 * 32;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)blockDim.x * gridDim.x) {
        Row32& w = dst[t >> 5];
        const int l = (int)(t & 31);
        if (t < n) {
            const uint64_t i = order ? order[t] : t;
            const DevBeam& b = beams[beam_of(beams, n_beams, i)];
            // the FP32 cosines normalised as the kernel would on load (m32::normalize)
            m32::Ray r{(float)(src.X[i] - b.origin[0]), (float)(src.Y[i] - b.origin[1]), (float)(src.Z[i] - b.origin[2]),
                       (float)src.cX[i], (float)src.cY[i], (float)src.cZ[i]};
            m32::normalize(r);
            w.X[l] = r.X;
            w.Y[l] = r.Y;
            w.Z[l] = r.Z;
            w.cX[l] = r.cX;
            w.cY[l] = r.cY;
            w.cZ[l] = r.cZ;
            w.lambda[l] = src.lambda[i];
            w.flag[l] = src.flag[i];
        } else {
            w.X[l] = w.Y[l] = w.Z[l] = w.cX[l] = w.cY[l] = w.cZ[l] = 0.0f;
            w.lambda[l] = 0.0;
            w.flag[l] = 0;
        }
    }
}

}  // namespace rtb
