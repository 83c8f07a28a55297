// engine.cuh -- host-side state and helpers of the C ABI.
#pragma once

#include <mutex>
#include <vector>

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

// Host-side scheme preparation (what the reference's host code computes
// before its launches).
struct PreparedScheme {
    DevScheme sch;
    std::vector<double> knots;
};

int prepare_surface(const rtb_surface& in, DevSurface& out, std::vector<double>& knots);
int prepare_scheme(const rtb_surface* s, size_t n, uint32_t fixes, int renorm_lost, PreparedScheme& out);
int surface_from_params(int cls, const double* params, DevSurface& s);
int add_table(const rtb_table* t, std::vector<double>& knots, int32_t& off, int32_t& cnt);
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
        cudaError_t e = cudaMallocAsync(&p, bytes ? bytes : 16, st);
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

}  // namespace rtb
