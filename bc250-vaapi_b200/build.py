"""Builds libb200enc.so (all CUDA kernels + the C-ABI) in-tree for sm_100a.

Invoked by __graft_entry__.build(); usable directly: python build.py [-v].
The .so lands in bc250-vaapi_b200/lib/ so it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib", "libb200enc.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["me.cu", "pframe.cu", "intra.cu", "deblock.cu", "gpu_compute_abi.cu", "noalloc.cu", "tc_gemm.cu", "proposal.cu", "proposal_infer.cu", "proposal_infer8.cu", "hevc.cu", "hevc_deblock.cu", "tune.cu", "batch.cu", "cavlc.cu", "t8x8.cu"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def build(verbose=False, force=False):
    srcs = sources()
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(HERE, "..", "include", f) for f in os.listdir(os.path.join(HERE, "..", "include"))]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    cmd = [NVCC, "-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-O3", "-shared",
           "-ccbin", "/usr/bin/g++", "-I" + os.path.join(HERE, "..", "include"),
           "-cudart", "static", "-o", LIB, *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(LIB)
