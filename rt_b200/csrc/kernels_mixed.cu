// kernels_mixed.cu -- the fused mixed-precision trace kernels for any scheme:
// FP64 ray state (k_fused_mixed, RTB_MIXED; mixed.cuh) and FP32 ray state
// (k_fused_mixed32, RTB_MIXED32; mixed32.cuh), each file holding its device
// code and precision choices.  Plans of a fixed scheme launch a specialised
// copy of the same code instead when one can be compiled at run time
// (jit.cpp).
#include "mixed32.cuh"

namespace rtb {

__global__ void __maxnreg__(64) k_fused_mixed(const DevScheme* __restrict__ g_sch, const double* knots,
                                              const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                              unsigned long long* counts, unsigned* err, int state_out,
                                              FrameArgs frame, TileSched ts) {
    fused_mixed<RtSurfaces>(g_sch, knots, beams, n_beams, in, out, counts, err, state_out, frame, ts);
}

__global__ void __maxnreg__(64) k_fused_mixed32(const DevScheme* __restrict__ g_sch, const double* knots,
                                                const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                                unsigned long long* counts, unsigned* err, int state_out,
                                                FrameArgs frame, TileSched ts) {
    fused_mixed32<Rt32Surfaces>(g_sch, knots, beams, n_beams, in, out, counts, err, state_out, frame, ts);
}

}  // namespace rtb
