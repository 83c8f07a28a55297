// kernels_mixed.cu -- fused mixed-precision trace kernel (see below).
#include "kernels.cuh"

namespace rtb {

__global__ void k_fused_mixed(const DevScheme*, const double*, const DevBeam*, int, DevRays, DevRays, unsigned long long*,
                              unsigned* err, int, FrameArgs) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, DEV_ERR_BAD_VALUE);
}

}  // namespace rtb
