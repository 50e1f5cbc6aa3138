"""Build the in-tree CUDA library xmcml_b200/libxmcml_b200.so for sm_100a.

Usage: python -m xmcml_b200.build [--force]

The library is one nvcc link of the CUDA transport kernel and the host C++ (device image, BVH,
XML/.surface/.mcml.out I/O, C-ABI). The FP32 walk is compiled with flush-to-zero and approximate
division and square root; the FP64 paths (edge-band triangle re-tests, near-critical Fresnel) are
unaffected by those flags.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libxmcml_b200.so")

SOURCES = ["transport.cu", "batch.cu", "surrogate.cu", "weight_table.cu", "noalloc.cu", "bvh_gpu.cu", "sparse_maps.cu",
           "capi.cpp", "io.cpp", "bvh.cpp"]
HEADERS = ["xmc_internal.h", "geom.cuh", "photon.cuh", "tc_gemm.cuh", "mlp_fused.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-ftz=true", "-prec-div=false", "-prec-sqrt=false", "-fmad=true",
    "-Xcompiler", "-fPIC,-O2",
    "-Xptxas", "-v",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "xmcml_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, f) for f in SOURCES]
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", "-o", tmp, *srcs,
           "-Xlinker", "-rpath,$ORIGIN", "-lcudart"]
    # host compiler: the system g++ (an environment CXX may lack OpenMP/specs)
    cmd[1:1] = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []
    proc = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    log = proc.stdout + proc.stderr
    with open(os.path.join(HERE, "build.log"), "w") as f:
        f.write(" ".join(cmd) + "\n" + log)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + log[-4000:])
    os.replace(tmp, LIB)
    if verbose:
        print(log)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
