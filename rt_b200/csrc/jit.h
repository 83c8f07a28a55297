// jit.h -- fused trace kernels specialised to a scheme's structure (jit.cpp).
#pragma once

#include <string>

#include "common.cuh"

namespace rtb {

// The CUDA source of the fused kernel of `precision` (RTB_MIXED, RTB_MIXED32
// or RTB_FP64)
// specialised to the structure of `sch` (one FixedShape per surface).
std::string scheme_source(const DevScheme& sch, int precision);

// NVRTC's version, or why it is unavailable (rtb_info).
std::string nvrtc_info();

// False when RTB_SPECIALIZE=0 is set in the environment.
bool specialize_enabled();

// Whether specialised kernels bake the surfaces' constants in (default), or
// only their structure (RTB_SPECIALIZE=structure).
bool bake_values();

// Compile (without loading) the specialised kernel: RTB_OK, or RTB_FAILED
// with `why`.  Needs no device.
int compile_scheme(const DevScheme& sch, int precision, std::string* why);

// The specialised kernel (compiled on first use when `compile`, then
// cached), as a function handle for cudaLaunchKernel; *kernel is NULL, and
// `why` says why, when NVRTC is unavailable or fails, or when the kernel was
// not compiled before and `compile` is false.  Error status only for CUDA
// errors of loading a compiled kernel.
int scheme_kernel(const DevScheme& sch, int precision, const void** kernel, std::string* why, bool compile = true);

// The adjoint's forward with checkpoints, its reverse sweep and its
// forward-mode sensitivities (adjoint_rev.cuh) compiled for the structure of
// `sch` (AdjShape per surface: kinds, classes, types fixed; transforms and
// all numbers read at run time, so the kernels serve every parameter value),
// compiled on first use and cached, as function handles for
// cudaLaunchKernel; all NULL, with `why`, when NVRTC is unavailable or
// fails.  Their parameters: (AdjArgs, DevRays in, counts, err), (AdjArgs,
// gX, gY, partial) and (AdjArgs, SurfD<1> table, dX, dY).
int adjoint_kernels(const DevScheme& sch, const void** forward, const void** reverse, const void** jvp,
                    std::string* why);

// The CUDA source of those kernels, and its compilation alone (no device).
std::string adjoint_source(const DevScheme& sch);
int compile_adjoint(const DevScheme& sch, std::string* why);

}  // namespace rtb
