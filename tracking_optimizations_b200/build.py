"""Build libgt.so (the sm_100a CUDA library behind include/gt.h) in-tree.

Run as ``python -m tracking_optimizations_b200.build`` or through
``__graft_entry__.build()``.  nvcc cross-compiles for sm_100a without a GPU.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgt.so")
SOURCES = ["gt_api.cu", "locate.cu", "locate_fast.cu", "finalize.cu", "link.cu", "assemble.cu", "noalloc.cu",
           "adjoint.cu", "synth.cu", "traj.cu", "ingest.cpp"]

# --fmad=false: the only fused multiply-adds are explicit fmaf() calls, so the
# kernels reproduce the oracle's operation order bit for bit.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-shared",
]


def nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def build(force=False, verbose=False):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    hdrs = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    hdrs += [os.path.join(ROOT, "include", h) for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h")]
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(s) <= t for s in srcs + hdrs):
            return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-I", CSRC,
                                   "-o", LIB + ".tmp"] + srcs + ["-lcudart", "-lz"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
