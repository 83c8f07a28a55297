"""Builds librtb200.so for sm_100a from rt_b200/csrc (nvcc, in tree).

The plain FP64 kernels are compiled with --fmad=false so that they round
every operation like the CPU oracle; the mixed-precision kernels keep FMA
contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librtb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
SOURCES = {
    "kernels_fp64.cu": ["--fmad=false"],
    "engine.cu": ["--fmad=false"],
    "trace.cu": ["--fmad=false"],
    "order.cu": [],
    "kernels_mixed.cu": ["--fmad=true"],
    "noalloc.cu": ["--fmad=false"],
    "plan.cu": ["--fmad=false"],
    "adjoint.cu": ["--fmad=false"],
    "scheme_xml.cpp": [],
    "reduce.cu": [],
    "io.cu": [],
    "jit.cpp": ["-I" + BUILD],
}

# Device sources compiled again at run time for scheme-specialised kernels
# (jit.cpp), by the names they are included under.
JIT_HEADERS = {
    "common.cuh": os.path.join(CSRC, "common.cuh"),
    "kernels.cuh": os.path.join(CSRC, "kernels.cuh"),
    "trace_common.cuh": os.path.join(CSRC, "trace_common.cuh"),
    "ray_fp64.cuh": os.path.join(CSRC, "ray_fp64.cuh"),
    "mixed.cuh": os.path.join(CSRC, "mixed.cuh"),
    "mixed32.cuh": os.path.join(CSRC, "mixed32.cuh"),
    "rowpipe.cuh": os.path.join(CSRC, "rowpipe.cuh"),
    "shape.cuh": os.path.join(CSRC, "shape.cuh"),
    "fused_fp64.cuh": os.path.join(CSRC, "fused_fp64.cuh"),
    "dual.cuh": os.path.join(CSRC, "dual.cuh"),
    "ray_ad.cuh": os.path.join(CSRC, "ray_ad.cuh"),
    "ray_rev.cuh": os.path.join(CSRC, "ray_rev.cuh"),
    "adjoint_rev.cuh": os.path.join(CSRC, "adjoint_rev.cuh"),
    "../../include/rtb.h": os.path.join(HERE, "..", "include", "rtb.h"),
}


def write_jit_headers() -> None:
    """_build/jit_headers.inc: the JIT_HEADERS as C++ raw string literals
    (rewritten only when they change)."""
    out = ["// generated by rt_b200/build.py from the device sources\n", "const JitHeader kJitHeaders[] = {\n"]
    for name, path in JIT_HEADERS.items():
        text = open(path).read()
        assert ')rtbjit"' not in text
        out.append(f'    {{"{name}", R"rtbjit({text})rtbjit"}},\n')
    out.append("};\n")
    body = "".join(out)
    path = os.path.join(BUILD, "jit_headers.inc")
    if not os.path.exists(path) or open(path).read() != body:
        with open(path, "w") as f:
            f.write(body)


def nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isabs(p) and os.path.exists(p) or not os.path.isabs(p)):
            return p
    return "nvcc"


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "rtb.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    write_jit_headers()
    objs = []
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _stale(o, s):
            cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_programs(verbose, force)
    return LIB


# Host programs over the C ABI (rt_b200/host/*.cpp -> rt_b200/bin/), linked
# against librtb200.so with a run path relative to the program.
PROGRAMS = ["rt_trace", "rt_ccd_frame", "rt_qe_comp", "rt_loss_comp", "rt_print_lambda"]
BIN = os.path.join(HERE, "bin")


def build_programs(verbose: bool = False, force: bool = False) -> None:
    os.makedirs(BIN, exist_ok=True)
    for name in PROGRAMS:
        src = os.path.join(HERE, "host", name + ".cpp")
        out = os.path.join(BIN, name)
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(
                os.path.getmtime(src), os.path.getmtime(LIB)):
            continue
        cmd = [nvcc(), "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", src, "-I" + os.path.join(HERE, "..", "include"), "-L" + HERE,
               "-lrtb200", "-lcudart", "-Xlinker", "-rpath,$ORIGIN/..", "-o", out]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
