// kernels_mixed.cu -- the fused mixed-precision trace kernel for any scheme
// (mixed.cuh holds its device code and the precision choices).  Plans of a
// fixed scheme launch a specialised copy of the same code instead when one
// can be compiled at run time (jit.cpp).
#include "mixed.cuh"

namespace rtb {

__global__ void __maxnreg__(64) k_fused_mixed(const DevScheme* __restrict__ g_sch, const double* knots,
                                              const DevBeam* beams, int n_beams, DevRays in, DevRays out,
                                              unsigned long long* counts, unsigned* err, int state_out,
                                              FrameArgs frame, TileSched ts) {
    fused_mixed<RtSurfaces>(g_sch, knots, beams, n_beams, in, out, counts, err, state_out, frame, ts);
}

}  // namespace rtb
