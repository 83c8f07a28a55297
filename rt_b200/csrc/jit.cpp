// jit.cpp -- copies of the fused trace kernels specialised to one scheme's
// structure, compiled at run time with NVRTC for plans.
//
// The generic fused kernels (k_fused_mixed, k_fused_fp64) read each surface's
// structure -- its intersection algorithm, type, class, aperture shape, which
// rotations apply, the number of polynomial terms -- from the scheme in
// shared memory and branch on it, surface by surface, in a loop.  A plan
// traces one scheme many times, so when it is made the same device code
// (mixed.cuh, fused_fp64.cuh) is compiled once more with the scheme's
// structure fixed: one call per surface with that surface's FixedShape, the
// untaken branches and polynomial loop bounds folded away.  The surfaces'
// numbers (curvatures, distances, angles, tables) are still read from the
// scheme at run time, so one compiled kernel serves every scheme of the same
// structure; kernels are cached by their source for the life of the process.
// The FP64 copy is compiled with --fmad=false like k_fused_fp64 and executes
// the same IEEE operations in the same order: its results are bit-identical.
//
// The device sources are built into the library (jit_headers.inc, generated
// from rt_b200/csrc and include/ at build time).  libnvrtc is opened at run
// time; without it, or with RTB_SPECIALIZE=0 in the environment, plans launch
// the generic kernels.
#include <dlfcn.h>
#include <nvrtc.h>

#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine.cuh"
#include "jit.h"

namespace rtb {
namespace {

struct JitHeader {
    const char* name;
    const char* text;
};

#include "jit_headers.inc"  // kJitHeaders[]: the device sources, by the names they are included as

// <cstdint>, <stdint.h>, <stddef.h> and <cuda_runtime.h> as the device code
// needs them (NVRTC has no system headers): the LP64 types of the host.
const char* const kTypes =
    "#pragma once\n"
    "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long int64_t;\n"
    "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
    "typedef unsigned long uint64_t; typedef unsigned long size_t; typedef long ptrdiff_t;\n";

const char* const kMixedName = "rtb_fused_mixed_scheme";
const char* const kMixed32Name = "rtb_fused_mixed32_scheme";
const char* const kFp64Name = "rtb_fused_fp64_scheme";

const char* kernel_name(int precision) {
    return precision == RTB_MIXED ? kMixedName : precision == RTB_MIXED32 ? kMixed32Name : kFp64Name;
}

struct Nvrtc {
    bool ok = false;
    std::string why;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    int major = 0, minor = 0;
};

Nvrtc load_nvrtc() {
    Nvrtc n;
    void* h = nullptr;
    for (const char* name : {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"}) {
        h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
        if (h) break;
    }
    if (!h) {
        n.why = "libnvrtc not found";
        return n;
    }
    n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
    auto version = reinterpret_cast<decltype(&nvrtcVersion)>(dlsym(h, "nvrtcVersion"));
    if (version) version(&n.major, &n.minor);
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    if (!n.ok) n.why = "libnvrtc lacks a function";
    return n;
}

const Nvrtc& nvrtc() {
    static const Nvrtc n = load_nvrtc();
    return n;
}

std::mutex g_mu;
std::map<std::string, std::vector<char>> g_cubins;  // compiled kernels, by source
std::map<std::string, cudaKernel_t> g_kernels;      // loaded kernels, by source

int compile_to_cubin(const std::string& src, bool fmad, std::vector<char>& cubin, std::string& log) {
    Range range("NVRTC compile");
    const Nvrtc& n = nvrtc();
    std::vector<const char*> names, texts;
    for (const char* t : {"cstdint", "stdint.h", "stddef.h"}) {
        names.push_back(t);
        texts.push_back(kTypes);
    }
    names.push_back("cuda_runtime.h");
    texts.push_back("#pragma once\n");
    for (const JitHeader& h : kJitHeaders) {
        names.push_back(h.name);
        texts.push_back(h.text);
    }
    nvrtcProgram prog = nullptr;
    if (n.create(&prog, src.c_str(), "rtb_fused_scheme.cu", (int)names.size(), texts.data(), names.data()) !=
        NVRTC_SUCCESS)
        return RTB_FAILED;
    // the options of kernels_mixed.cu (FMA contraction) or kernels_fp64.cu
    // (none); -default-device: the host function declarations of the headers
    // are compiled as (unused) device functions
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", fmad ? "--fmad=true" : "--fmad=false",
                          "-lineinfo", "-default-device"};
    nvrtcResult r = n.compile(prog, (int)(sizeof(opts) / sizeof(opts[0])), opts);
    size_t ls = 0;
    if (n.log_size(prog, &ls) == NVRTC_SUCCESS && ls > 1) {
        log.resize(ls);
        n.log(prog, &log[0]);
    }
    size_t cs = 0;
    if (r == NVRTC_SUCCESS && n.cubin_size(prog, &cs) == NVRTC_SUCCESS && cs > 0) {
        cubin.resize(cs);
        if (n.cubin(prog, cubin.data()) != NVRTC_SUCCESS) cubin.clear();
    }
    n.destroy(&prog);
    return cubin.empty() ? RTB_FAILED : RTB_OK;
}

}  // namespace

// FixedShape<...> of surface s: the fields RtShape reads.
static std::string fixed_shape(const DevSurface& s) {
    char t[200];
    std::snprintf(t, sizeof(t), "FixedShape<%d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d>", (int)s.kind,
                  (int)s.type, (int)s.cls, (int)s.shape, (int)s.gr_type, s.translate != 0 ? 1 : 0, (int)s.rot_mask,
                  (int)s.n_poly, s.non_aux != 0 ? 1 : 0, s.sag_cull != 0 ? 1 : 0, s.c == 0.0 ? 1 : 0,
                  s.rot32 != 0 ? 1 : 0, s.first32 != 0 ? 1 : 0);
    return t;
}

static const char* const kParams =
    "        const rtb::DevScheme* __restrict__ g_sch, const double* knots, const rtb::DevBeam* beams,\n"
    "        int n_beams, rtb::DevRays in, rtb::DevRays out, unsigned long long* counts, unsigned* err,\n"
    "        int state_out, rtb::FrameArgs frame, rtb::TileSched ts) {\n";

// The surfaces' constants baked into the kernel: a __constant__ image of
// sch.s[0 .. n_surfaces), which the surface code reads at addresses known at
// compile time -- constant-bank operands of its instructions instead of
// shared-memory loads and their address arithmetic.  The run time fields of
// the scheme (the knot tables, the beams) are read as before.
static std::string surface_constants(const DevScheme& sch) {
    static_assert(sizeof(DevSurface) % 8 == 0, "DevSurface is baked as 64-bit words");
    const size_t words = (size_t)sch.n_surfaces * sizeof(DevSurface) / 8;
    std::vector<unsigned long long> w(words);
    std::memcpy(w.data(), sch.s, words * 8);
    std::string t = "namespace rtb {\nstatic __constant__ const unsigned long long k_surface_words[" +
                    std::to_string(words) + "] = {";
    char buf[32];
    for (size_t i = 0; i < words; ++i) {
        std::snprintf(buf, sizeof(buf), "%s0x%llxull", (i % 6) ? ", " : ",\n    ", w[i]);
        t += (i == 0) ? buf + 1 : buf;
    }
    t += "};\n__device__ __forceinline__ const DevSurface* k_surfaces() {\n"
         "    return reinterpret_cast<const DevSurface*>(k_surface_words);\n}\n"
         "constexpr uint32_t k_fixes = " + std::to_string(sch.fixes) + "u;\n}  // namespace rtb\n";
    return t;
}

// Register cap of the specialised kernels: 64 (32 warps per SM), or
// RTB_JIT_MAXNREG (32..128) to measure other occupancies.
static std::string jit_maxnreg() {
    const char* e = std::getenv("RTB_JIT_MAXNREG");
    const int v = e ? std::atoi(e) : 0;
    return std::to_string((v >= 32 && v <= 128) ? v : 64);
}

std::string scheme_source(const DevScheme& sch, int precision) {
    std::string src;
    const std::string maxnreg = jit_maxnreg();
    const bool bake = bake_values();
    const std::string S = bake ? "k_surfaces()[" : "sch->s[";
    const std::string F = bake ? "k_fixes" : "sch->fixes";
    if (precision == RTB_MIXED) {
        src = "#include \"mixed.cuh\"\n" + (bake ? surface_constants(sch) : std::string()) +
              "namespace rtb {\n"
              "struct SchemeSurfaces {\n"
              "    __device__ __forceinline__ static void run(const DevScheme* sch, const double* knots,\n"
              "        const BeamCtx& bc, double lam, mx::TableMemo& memo, mx::Ray& r, int& stage) {\n";
        for (int k = 0; k < sch.n_surfaces; ++k) {
            const std::string ks = std::to_string(k);
            src += "        if (stage == -1) stage = mx_surface<" + fixed_shape(sch.s[k]) + ">(" + S + ks + "], " +
                   ks + ", " + F + ", knots, bc, lam, memo, r);\n";
        }
        src += std::string("    }\n};\n}  // namespace rtb\n"
                           "extern \"C\" __global__ void __maxnreg__(" + maxnreg + ") ") + kMixedName + "(\n" + kParams +
               "    rtb::fused_mixed<rtb::SchemeSurfaces>(g_sch, knots, beams, n_beams, in, out, counts, err,\n"
               "                                        state_out, frame, ts);\n}\n";
    } else if (precision == RTB_MIXED32) {
        src = "#include \"mixed32.cuh\"\n" + (bake ? surface_constants(sch) : std::string()) +
              "namespace rtb {\n"
              "struct SchemeSurfaces32 {\n"
              "    __device__ __forceinline__ static void run(const DevScheme* sch, const double* knots,\n"
              "        const BeamCtx& bc, const double* off0, double lam, mx::TableMemo& memo, m32::Ray& r,\n"
              "        mx::Ray& q, int& stage) {\n";
        for (int k = 0; k < sch.n_surfaces; ++k) {
            if (!sch.s[k].non_aux) continue;  // folded into the next surface's transform
            const std::string ks = std::to_string(k);
            src += "        if (stage == -1) stage = m32_surface<" + fixed_shape(sch.s[k]) + ">(" + S + ks + "], " +
                   ks + ", " + F + ", knots, bc, off0, lam, memo, r, q);\n";
        }
        src += std::string("    }\n};\n}  // namespace rtb\n"
                           "extern \"C\" __global__ void __maxnreg__(" + maxnreg + ") ") + kMixed32Name + "(\n" + kParams +
               "    rtb::fused_mixed32<rtb::SchemeSurfaces32>(g_sch, knots, beams, n_beams, in, out, counts, err,\n"
               "                                            state_out, frame, ts);\n}\n";
    } else {
        src = "#include \"fused_fp64.cuh\"\n" + (bake ? surface_constants(sch) : std::string()) +
              "namespace rtb {\n"
              "struct SchemeSurfacesF64 {\n"
              "    __device__ __forceinline__ static void run(const DevScheme* sch, const double* knots,\n"
              "        const DevBeam* beams, int b, double lam, unsigned* err, f64::Ray& r, int& stage) {\n";
        for (int k = 0; k < sch.n_surfaces; ++k) {
            const std::string ks = std::to_string(k);
            src += "        if (stage == -1) f64_surface<" + fixed_shape(sch.s[k]) + ">(" + S + ks + "], " + ks + ", " +
                   F + ", knots, beams, b, lam, err, r, stage);\n        __syncthreads();\n";
        }
        src += std::string("    }\n};\n}  // namespace rtb\n"
                           "extern \"C\" __global__ void __maxnreg__(" + maxnreg + ") ") + kFp64Name + "(\n" + kParams +
               "    rtb::fused_fp64<rtb::SchemeSurfacesF64>(g_sch, knots, beams, n_beams, in, out, counts, err,\n"
               "                                          state_out, frame, ts);\n}\n";
    }
    return src;
}

std::string nvrtc_info() {
    const Nvrtc& n = nvrtc();
    if (!n.ok) return "unavailable (" + n.why + ")";
    return std::to_string(n.major) + "." + std::to_string(n.minor) +
           (specialize_enabled() ? "" : " (RTB_SPECIALIZE=0)");
}

bool bake_values() {
    const char* e = std::getenv("RTB_SPECIALIZE");
    return !(e && std::strcmp(e, "structure") == 0);
}

bool specialize_enabled() {
    const char* e = std::getenv("RTB_SPECIALIZE");
    return !(e && std::strcmp(e, "0") == 0);
}

// Optional on-disk cache of compiled kernels, for processes that trace the
// same scheme structures (RTB_JIT_CACHE=<directory>; off when unset or
// empty).  A file holds its full key -- NVRTC's version, the options, the
// device sources and the kernel's source -- and the cubin, and is used only
// when that key equals this build's exactly.  Files are written under a
// temporary name and renamed into place, so that a reader never sees half a
// file.
static std::string cache_dir() {
    const char* e = std::getenv("RTB_JIT_CACHE");
    return (e && *e) ? std::string(e) : std::string();
}

static std::string cache_key(const std::string& src, bool fmad) {
    const Nvrtc& n = nvrtc();
    std::string k = "rtb-jit 1\nnvrtc " + std::to_string(n.major) + "." + std::to_string(n.minor) +
                    (fmad ? " fmad\n" : " no-fmad\n");
    for (const JitHeader& h : kJitHeaders) {
        k += h.name;
        k += '\n';
        k += h.text;
        k += '\n';
    }
    return k + src;
}

static std::string cache_path(const std::string& dir, const std::string& key) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : key) h = (h ^ c) * 1099511628211ull;
    char name[40];
    std::snprintf(name, sizeof(name), "/rtb-%016llx.cubin", (unsigned long long)h);
    return dir + name;
}

static bool disk_load(const std::string& dir, const std::string& key, std::vector<char>& cubin) {
    std::ifstream f(cache_path(dir, key), std::ios::binary);
    uint64_t kn = 0, cn = 0;
    if (!f.read(reinterpret_cast<char*>(&kn), 8) || kn != key.size()) return false;
    std::string k(kn, '\0');
    if (!f.read(&k[0], (std::streamsize)kn) || k != key) return false;
    if (!f.read(reinterpret_cast<char*>(&cn), 8) || cn == 0 || cn > (1ull << 30)) return false;
    cubin.resize(cn);
    return (bool)f.read(cubin.data(), (std::streamsize)cn);
}

static void disk_store(const std::string& dir, const std::string& key, const std::vector<char>& cubin) {
    const std::string path = cache_path(dir, key);
    const std::string tmp = path + ".tmp." + std::to_string((long long)getpid());
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        const uint64_t kn = key.size(), cn = cubin.size();
        f.write(reinterpret_cast<const char*>(&kn), 8);
        f.write(key.data(), (std::streamsize)kn);
        f.write(reinterpret_cast<const char*>(&cn), 8);
        f.write(cubin.data(), (std::streamsize)cn);
        if (!f) {
            f.close();
            std::remove(tmp.c_str());
            return;
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

// The compiled kernel for `src` (g_mu held): from memory, else from the
// disk cache, else compiled (when `compile`).
static const std::vector<char>* cubin_for(const std::string& src, bool fmad, std::string* why, bool compile) {
    auto it = g_cubins.find(src);
    if (it != g_cubins.end()) return &it->second;
    const std::string dir = nvrtc().ok ? cache_dir() : std::string();
    const std::string key = dir.empty() ? std::string() : cache_key(src, fmad);
    if (!dir.empty()) {
        std::vector<char> cubin;
        if (disk_load(dir, key, cubin)) return &g_cubins.emplace(src, std::move(cubin)).first->second;
    }
    if (!compile) {
        if (why) *why = "not compiled yet";
        return nullptr;
    }
    const Nvrtc& n = nvrtc();
    if (!n.ok) {
        if (why) *why = n.why;
        return nullptr;
    }
    std::vector<char> cubin;
    std::string log;
    if (compile_to_cubin(src, fmad, cubin, log) != RTB_OK) {
        if (why) *why = "NVRTC failed: " + log.substr(0, 2000);
        return nullptr;
    }
    if (!dir.empty()) disk_store(dir, key, cubin);
    return &g_cubins.emplace(src, std::move(cubin)).first->second;
}

int compile_scheme(const DevScheme& sch, int precision, std::string* why) {
    std::lock_guard<std::mutex> g(g_mu);
    return cubin_for(scheme_source(sch, precision), precision != RTB_FP64, why, true) ? RTB_OK : RTB_FAILED;
}

// Load the kernel `name` of `src` (compiled when needed and `compile`).
static int load_kernel(const std::string& src, bool fmad, const char* name, const void** kernel, std::string* why,
                       bool compile) {
    *kernel = nullptr;
    std::lock_guard<std::mutex> g(g_mu);
    const std::string kkey = src + '\0' + name;  // a source may hold several kernels
    auto it = g_kernels.find(kkey);
    if (it != g_kernels.end()) {
        *kernel = reinterpret_cast<const void*>(it->second);
        return RTB_OK;
    }
    cudaLibrary_t lib = nullptr;
    cudaKernel_t k = nullptr;
    cudaError_t e = cudaSuccess;
    for (int attempt = 0; attempt < 2; ++attempt) {
        const std::vector<char>* cubin = cubin_for(src, fmad, why, compile);
        if (!cubin) return RTB_OK;
        lib = nullptr;
        e = cudaLibraryLoadData(&lib, cubin->data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
        if (e == cudaSuccess) e = cudaLibraryGetKernel(&k, lib, name);
        if (e == cudaSuccess) break;
        if (lib) cudaLibraryUnload(lib);
        // a cubin that does not load (a damaged cache file): compile afresh once
        g_cubins.erase(src);
        const std::string dir = cache_dir();
        if (!dir.empty()) std::remove(cache_path(dir, cache_key(src, fmad)).c_str());
        if (!compile) break;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();  // handled here: not to be reported by a later launch check
        if (!compile) return RTB_OK;  // one-shot traces run the generic kernel
        return cuda_status(e);
    }
    g_kernels.emplace(kkey, k);
    *kernel = reinterpret_cast<const void*>(k);
    return RTB_OK;
}

int scheme_kernel(const DevScheme& sch, int precision, const void** kernel, std::string* why, bool compile) {
    return load_kernel(scheme_source(sch, precision), precision != RTB_FP64, kernel_name(precision), kernel, why,
                       compile);
}

// AdjShape<...> of surface s (adjoint_rev.cuh).
static std::string adj_shape(const DevSurface& s) {
    char t[160];
    std::snprintf(t, sizeof(t), "AdjShape<%d, %d, %d, %d, %d, %d, %d, %d>", (int)s.kind, (int)s.type, (int)s.cls,
                  (int)s.shape, (int)s.gr_type, (int)s.n_poly, s.non_aux != 0 ? 1 : 0, s.c == 0.0 ? 1 : 0);
    return t;
}

static const char* const kAdjForwardName = "rtb_adj_forward_scheme";
static const char* const kAdjReverseName = "rtb_adj_reverse_scheme";
static const char* const kAdjJvpName = "rtb_adj_jvp_scheme";

std::string adjoint_source(const DevScheme& sch) {
    std::string src =
        "#include \"adjoint_rev.cuh\"\n"
        "namespace rtb {\n"
        "struct SchemeAdjForward {\n"
        "    __device__ __forceinline__ static int run(const AdjArgs& a, size_t i, int b, double lam, unsigned* err,\n"
        "                                              f64::Ray& r) {\n"
        "        int stage = -1;\n";
    for (int k = 0; k < sch.n_surfaces; ++k)
        src += "        if (stage == -1) stage = fwd_surface<" + adj_shape(sch.s[k]) + ">(a, " + std::to_string(k) +
               ", i, b, lam, err, r);\n";
    src += "        return stage;\n    }\n};\n"
           "struct SchemeAdjJvp {\n"
           "    __device__ __forceinline__ static void run(const AdjArgs& a, const ad::SurfD<1>* table, int b,\n"
           "                                               double lam, ad::RayD<1>& r) {\n";
    for (int k = 0; k < sch.n_surfaces; ++k)
        src += "        jvp_surface<" + adj_shape(sch.s[k]) + ">(a, " + std::to_string(k) + ", table, b, lam, r);\n";
    src += "    }\n};\n"
           "struct SchemeAdjSurfaces {\n"
           "    __device__ __forceinline__ static void sweep(const AdjArgs& a, RevRay& ray, int lane, double* acc_row) {\n";
    for (int k = sch.n_surfaces - 1; k >= 0; --k)
        src += "        rev_surface<" + adj_shape(sch.s[k]) + ">(a, " + std::to_string(k) + ", ray, lane, acc_row);\n";
    src += std::string("    }\n};\n}  // namespace rtb\n"
                       "extern \"C\" __global__ void __launch_bounds__(256) ") + kAdjForwardName +
           "(rtb::AdjArgs a, rtb::DevRays in,\n        unsigned long long* counts, unsigned* err) {\n"
           "    rtb::adj_forward<rtb::SchemeAdjForward>(a, in, counts, err);\n}\n"
           "extern \"C\" __global__ void __launch_bounds__(rtb::kAdjThreads, 4) " + kAdjReverseName +
           "(rtb::AdjArgs a,\n        const double* gX, const double* gY, double* partial) {\n"
           "    rtb::adj_reverse<rtb::SchemeAdjSurfaces>(a, gX, gY, partial);\n}\n"
           "extern \"C\" __global__ void __launch_bounds__(rtb::kAdjThreads) " + kAdjJvpName +
           "(rtb::AdjArgs a,\n        const rtb::ad::SurfD<1>* table, double* dX, double* dY) {\n"
           "    rtb::adj_jvp<rtb::SchemeAdjJvp>(a, table, dX, dY);\n}\n";
    return src;
}

int adjoint_kernels(const DevScheme& sch, const void** forward, const void** reverse, const void** jvp,
                    std::string* why) {
    const std::string src = adjoint_source(sch);
    *reverse = *jvp = nullptr;
    int st = load_kernel(src, false, kAdjForwardName, forward, why, true);
    if (st != RTB_OK || !*forward) return st;
    st = load_kernel(src, false, kAdjReverseName, reverse, why, true);
    if (st == RTB_OK && *reverse) st = load_kernel(src, false, kAdjJvpName, jvp, why, true);
    if (!*reverse || !*jvp) *forward = *reverse = *jvp = nullptr;
    return st;
}

int compile_adjoint(const DevScheme& sch, std::string* why) {
    std::lock_guard<std::mutex> g(g_mu);
    return cubin_for(adjoint_source(sch), false, why, true) ? RTB_OK : RTB_FAILED;
}

}  // namespace rtb

using namespace rtb;

int rtb_specialize(const rtb_surface* surfaces, size_t n_surfaces, uint32_t fixes, int32_t precision, char* note,
                   size_t note_len) {
    if (note && note_len > 0) note[0] = 0;
    if (precision != RTB_FP64 && precision != RTB_MIXED && precision != RTB_MIXED32) return RTB_BAD_VALUE;
    PreparedScheme ps;
    int st = prepare_scheme(surfaces, n_surfaces, fixes, 0, ps);
    if (st != RTB_OK) return st;
    std::string why;
    st = compile_scheme(ps.sch, precision, &why);
    if (note && note_len > 0) std::snprintf(note, note_len, "%s", why.c_str());
    return st;
}

int rtb_adjoint_specialize(const rtb_surface* surfaces, size_t n_surfaces, uint32_t fixes, char* note,
                           size_t note_len) {
    if (note && note_len > 0) note[0] = 0;
    PreparedScheme ps;
    int st = prepare_scheme(surfaces, n_surfaces, fixes, 0, ps);
    if (st != RTB_OK) return st;
    std::string why;
    st = compile_adjoint(ps.sch, &why);
    if (note && note_len > 0) std::snprintf(note, note_len, "%s", why.c_str());
    return st;
}
