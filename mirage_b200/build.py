"""Build recipe for the in-tree native library (libmirage_b200.so) and the mirage_gpu tool.

nvcc cross-compiles for sm_100a without a GPU; the library links the CUDA runtime statically
so the built .so travels to a GPU host as one file.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmirage_b200.so")
TOOL = os.path.join(HERE, "mirage_gpu")
LOADGEN = os.path.join(HERE, "libmg_loadgen.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: the score arithmetic must round exactly as the reference's separate IEEE ops.
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2,-fno-fast-math",
          "-Xcompiler", "-ffp-contract=off"]

LIB_SOURCES = ["mg_lib.cu", "mg_server.cu", "mhm.cpp", "mg_output.cu", "mg_noalloc.cu", "mg_build.cu", "mg_parse.cu",
               "mg_pack.cpp"]
HEADERS = ["mg_device.cuh", "mg_kernels.cuh", "mg_lean.cuh", "mg_dual.cuh", "mg_long.cuh", "mhm.h", "mg_internal.h",
           "mg_ring.h", "mg_pack.h"]
TOOL_SOURCES = ["mirage_gpu.cpp"]
LOADGEN_SOURCES = ["mg_loadgen.cpp"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    inc = os.path.join(os.path.dirname(HERE), "include")
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = srcs + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(inc, "mirage_b200.h")]
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    if force or _stale(LIB, deps):
        objs = []
        for s in srcs:
            o = os.path.join(objdir, os.path.basename(s) + ".o")
            if force or _stale(o, [s] + deps[len(srcs):]):
                cmd = [NVCC, *ARCH, *COMMON, "-I", inc, "-c", s, "-o", o]
                if verbose:
                    print(" ".join(cmd), flush=True)
                subprocess.run(cmd, check=True)
            objs.append(o)
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lpthread"]
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    tsrc = [os.path.join(CSRC, s) for s in TOOL_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if tsrc and (force or _stale(TOOL, tsrc + [LIB])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", inc, *tsrc, "-o", TOOL, "-L", HERE, "-lmirage_b200",
               "-Wl,-rpath,$ORIGIN", "-lpthread"]
        subprocess.run(cmd, check=True)
    lsrc = [os.path.join(CSRC, s) for s in LOADGEN_SOURCES]
    if force or _stale(LOADGEN, lsrc + [LIB, os.path.join(inc, "mirage_b200.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", inc, *lsrc, "-o", LOADGEN, "-L", HERE,
               "-lmirage_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
