"""Build libvlsgpu.so (sm_100a) in-tree with nvcc.

FP64 parity with the reference's double-precision rules needs IEEE division
and square root (nvcc defaults) and no multiply-add contraction, hence
-fmad=false on the device and -ffp-contract=off on the host.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvlsgpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
SOURCES = ["vlsg_api.cu"]
HEADERS = ["vlsg_common.cuh", "vlsg_passes.cuh", "vlsg_frontier.cuh", "vlsg_rates.cuh",
           "vlsg_maint.cuh", "vlsg_scan.cuh", "vlsg_exchange.cuh", "vlsg_metrics.cuh",
           "vlsg_engine.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "--expt-relaxed-constexpr",
    "-shared",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "vlsg.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-I", INCLUDE] + \
          [os.path.join(CSRC, s) for s in SOURCES] + ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
