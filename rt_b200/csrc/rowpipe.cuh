// rowpipe.cuh -- the fused mixed kernels' ray input: rows of 32 rays staged
// in shared memory by bulk asynchronous copies.
//
// A plan keeps its rays in tracing order as row blocks: 32 consecutive rays,
// each component stored for the 32 rays in turn, then their flags -- Row64
// (FP64 X..cZ and wavelength, 1824 bytes) or Row32 (FP32 position relative
// to the beam's origin and direction, FP64 wavelength, 1056 bytes).  A warp
// traces one row at a time, one ray per lane.  Each warp owns one row buffer
// in shared memory: when a row has landed, every lane copies its ray into
// registers (conflict-free: lane l reads element l of each component), and
// one lane then starts the bulk copy of the warp's next row (cp.async.bulk
// global -> shared, its completion counted on the warp's mbarrier) into the
// same buffer, which lands while the warp traces the current row.  A row's
// loads thus cost one instruction per warp, issued a whole row of tracing
// ahead, instead of a scoreboard wait per lane and array.
//
// Rows are handed out as TileSched tiles of rpt rows.  A warp draws its tiles
// from the counter one tile ahead: the atomic that names the tile after next
// is issued when a tile starts and its result is first used when that tile
// ends, so its round trip to L2 is hidden behind a tile of tracing; the copy
// of the next tile's first row starts with the last row of the current one,
// as early as any other row's.
// Every wait on the mbarrier is bounded: past kWaitLimit polls the kernel
// raises DEV_ERR_TIMEOUT, waits (bounded again) for the copy it issued and
// stops taking rows.  The copies read this GPU's own memory only and use no
// cluster multicast.
#pragma once

#include "trace_common.cuh"

namespace rtb {

// Row blocks of 32 rays (device layout of the plans' tracing-order copies).
struct Row64 {
    double X[32], Y[32], Z[32], cX[32], cY[32], cZ[32], lambda[32];
    char flag[32];
};
struct Row32 {
    float X[32], Y[32], Z[32], cX[32], cY[32], cZ[32];  // position relative to the beam's origin; cosines
    double lambda[32];
    char flag[32];
};
static_assert(sizeof(Row64) % 16 == 0 && sizeof(Row32) % 16 == 0, "bulk copies move multiples of 16 bytes");

// Bytes of one warp's row buffer: the row and the mbarrier.
template <class Row>
__host__ __device__ constexpr unsigned row_buffer_bytes() {
    return ((unsigned)sizeof(Row) + 8u + 127u) / 128u * 128u;
}

constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    // make the initialised barrier visible to the asynchronous proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One elected lane: expect the row's bytes on the barrier and start its copy.
__device__ __forceinline__ void row_copy(uint32_t bar, uint32_t dst, const void* src, unsigned bytes) {
    // the lanes' reads of the previous row (generic proxy) come before the
    // asynchronous writes of this one
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Poll the barrier's phase `parity` at most kWaitLimit times.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (unsigned i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2; selp.b32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

// The rows of one warp.  Usage, per row:
//   while (rows.begin()) {            // waits for the row (row-block inputs)
//       ... lane reads its ray (rows.row<Row>(), or the SoA arrays at rows.slot())
//       rows.prefetch();              // starts the copy of the next row into the same buffer
//       ... traces it
//   }
struct RowLoop {
    const TileSched& ts;
    uint64_t n, n_tiles;
    uint64_t tile = 0, next_tile_ = 0;
    unsigned long long ahead = 0;  // lane 0: the counter value drawn for the tile after next
    int j = 0, next_j = 0;
    bool have_next = false, packed;
    unsigned row_bytes;
    unsigned char* buf = nullptr;
    uint32_t bar = 0, parity = 0;
    unsigned* err;

    __device__ RowLoop(const TileSched& t, uint64_t n_rays, unsigned char* warp_buf, unsigned row_size, unsigned* e)
        : ts(t), n(n_rays), packed(t.rows != nullptr), row_bytes(row_size), buf(warp_buf), err(e) {
        const uint64_t rows = (n + 31) / 32;
        n_tiles = (rows + (uint64_t)ts.rpt - 1) / (uint64_t)ts.rpt;
        if (packed) {
            bar = smem_addr(buf + ((row_bytes + 7u) & ~7u));
            if ((threadIdx.x & 31) == 0) mbar_init(bar);
            __syncwarp();
        }
        have_next = next_tile(ts, n_tiles, next_tile_);
        next_j = 0;
        if (have_next) {
            issue(next_tile_, 0);
            draw_ahead();
        }
    }
    // Lane 0 draws a tile from the counter; the result is read at the next
    // tile switch (take_ahead).
    __device__ void draw_ahead() {
        if ((threadIdx.x & 31) == 0) ahead = atomicAdd(ts.next, 1ull);
    }
    __device__ bool take_ahead(uint64_t& t) const {
        t = __shfl_sync(0xffffffffu, ahead, 0);
        return t < n_tiles;
    }
    __device__ uint64_t row_of(uint64_t t, int jj) const { return t * (uint64_t)ts.rpt + (uint64_t)jj; }
    __device__ void issue(uint64_t t, int jj) {
        if (!packed) return;
        if ((threadIdx.x & 31) == 0)
            row_copy(bar, smem_addr(buf), static_cast<const unsigned char*>(ts.rows) + row_of(t, jj) * row_bytes,
                     row_bytes);
    }
    // Start the next row: false when the warp has no rows left (or a copy
    // never completed).
    __device__ bool begin() {
        if (!have_next) return false;
        tile = next_tile_;
        j = next_j;
        if (packed) {
            bool ok = mbar_wait(bar, parity);
            parity ^= 1u;
            if (!__all_sync(0xffffffffu, ok)) {
                if ((threadIdx.x & 31) == 0) atomicOr(err, (unsigned)DEV_ERR_TIMEOUT);
                mbar_wait(bar, parity ^ 1u);  // the copy in flight, once more (bounded)
                have_next = false;
                return false;
            }
        }
        return true;
    }
    // The row after the current one: the next row of the tile, or the first
    // row of the warp's next tile; its copy starts now.  Call once per row,
    // after every lane has read its record.
    __device__ void prefetch() {
        __syncwarp();
        if (j + 1 < ts.rpt && row_of(tile, j + 1) * 32 < n) {
            next_tile_ = tile;
            next_j = j + 1;
            have_next = true;
        } else {
            have_next = take_ahead(next_tile_);
            next_j = 0;
            if (have_next) draw_ahead();
        }
        if (have_next) issue(next_tile_, next_j);
    }
    __device__ uint64_t slot() const { return row_of(tile, j) * 32 + (threadIdx.x & 31); }
    template <class Row>
    __device__ const Row& row() const {
        return *reinterpret_cast<const Row*>(buf);
    }
};

// Shared memory of the row buffers of a block of `threads` threads.
template <class Row>
__host__ __device__ constexpr size_t row_buffers_bytes(int threads) {
    return (size_t)(threads / 32) * row_buffer_bytes<Row>();
}

// This warp's row buffer: after the scheme and its tables in the fused
// kernels' dynamic shared memory.
template <class Row>
__device__ __forceinline__ unsigned char* warp_row_buffer(int n_knots) {
    extern __shared__ __align__(16) unsigned char smem[];
    const size_t base = (((sizeof(DevScheme) + 15) / 16) * 16 + sizeof(double) * (size_t)n_knots + 127) / 128 * 128;
    return smem + base + (size_t)(threadIdx.x >> 5) * row_buffer_bytes<Row>();
}

}  // namespace rtb
