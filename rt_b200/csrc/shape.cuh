// shape.cuh -- the structure of a surface as its device code reads it.
#pragma once

#include "common.cuh"

namespace rtb {

// The structure of a surface -- what its code branches on -- read from its
// DevSurface at run time (RtShape), or fixed at compile time (FixedShape) for
// a kernel specialised to one scheme, where the untaken branches and the
// polynomial loops' bounds fold away.
struct RtShape {
    __device__ __forceinline__ static int kind(const DevSurface& s) { return s.kind; }
    __device__ __forceinline__ static int type(const DevSurface& s) { return s.type; }
    __device__ __forceinline__ static int cls(const DevSurface& s) { return s.cls; }
    __device__ __forceinline__ static int shape(const DevSurface& s) { return s.shape; }
    __device__ __forceinline__ static int gr_type(const DevSurface& s) { return s.gr_type; }
    __device__ __forceinline__ static bool translate(const DevSurface& s) { return s.translate != 0; }
    __device__ __forceinline__ static int rot_mask(const DevSurface& s) { return s.rot_mask; }
    __device__ __forceinline__ static int n_poly(const DevSurface& s) { return s.n_poly; }
    __device__ __forceinline__ static bool non_aux(const DevSurface& s) { return s.non_aux != 0; }
    __device__ __forceinline__ static bool sag_cull(const DevSurface& s) { return s.sag_cull != 0; }
    __device__ __forceinline__ static bool poly_only(const DevSurface& s) { return s.c == 0.0; }
    __device__ __forceinline__ static bool rot32(const DevSurface& s) { return s.rot32 != 0; }
    __device__ __forceinline__ static bool first32(const DevSurface& s) { return s.first32 != 0; }
};

template <int KIND, int TYPE, int CLS, int SHAPE, int GRT, int TRANS, int ROT, int NPOLY, int NONAUX, int SAG,
          int POLYONLY, int ROT32 = 0, int FIRST32 = 0>
struct FixedShape {
    __device__ __forceinline__ static constexpr int kind(const DevSurface&) { return KIND; }
    __device__ __forceinline__ static constexpr int type(const DevSurface&) { return TYPE; }
    __device__ __forceinline__ static constexpr int cls(const DevSurface&) { return CLS; }
    __device__ __forceinline__ static constexpr int shape(const DevSurface&) { return SHAPE; }
    __device__ __forceinline__ static constexpr int gr_type(const DevSurface&) { return GRT; }
    __device__ __forceinline__ static constexpr bool translate(const DevSurface&) { return TRANS != 0; }
    __device__ __forceinline__ static constexpr int rot_mask(const DevSurface&) { return ROT; }
    __device__ __forceinline__ static constexpr int n_poly(const DevSurface&) { return NPOLY; }
    __device__ __forceinline__ static constexpr bool non_aux(const DevSurface&) { return NONAUX != 0; }
    __device__ __forceinline__ static constexpr bool sag_cull(const DevSurface&) { return SAG != 0; }
    __device__ __forceinline__ static constexpr bool poly_only(const DevSurface&) { return POLYONLY != 0; }
    __device__ __forceinline__ static constexpr bool rot32(const DevSurface&) { return ROT32 != 0; }
    __device__ __forceinline__ static constexpr bool first32(const DevSurface&) { return FIRST32 != 0; }
};

}  // namespace rtb
