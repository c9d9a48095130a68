"""Build libvlsgpu.so (sm_100a) in-tree with nvcc.

Three compilation units, compiled in parallel and linked into one library:
  vlsg_api.cu       the C ABI and the device comparison of two level sets;
  vlsg_engine64.cu  the FP64 engine -- parity with the reference's
                    double-precision rules needs IEEE division and square
                    root (nvcc defaults) and no multiply-add contraction,
                    hence -fmad=false (and -ffp-contract=off on the host);
  vlsg_engine32.cu  the FP32 engine, with multiply-add contraction (its
                    results are held to a tolerance against the FP64 path).
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvlsgpu.so")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
UNITS = {
    "vlsg_api.cu": ["-fmad=false"],
    "vlsg_engine64.cu": ["-fmad=false"],
    "vlsg_engine32.cu": ["-fmad=true"],
}
SOURCES = list(UNITS)
HEADERS = ["vlsg_common.cuh", "vlsg_iface.h", "vlsg_passes.cuh", "vlsg_frontier.cuh",
           "vlsg_rates.cuh", "vlsg_maint.cuh", "vlsg_scan.cuh", "vlsg_exchange.cuh",
           "vlsg_metrics.cuh", "vlsg_compare.cuh", "vlsg_velcb.cuh", "vlsg_voids.cuh", "vlsg_batch.cuh", "vlsg_engine.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "--expt-relaxed-constexpr",
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


def _compile(src, extra, verbose):
    obj = os.path.join(OBJ, src.replace(".cu", ".o"))
    cmd = [nvcc()] + NVCC_FLAGS + UNITS[src] + list(extra) + ["-I", INCLUDE, "-c",
                                                              os.path.join(CSRC, src), "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    return obj, r


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(len(UNITS)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose), SOURCES))
    for obj, r in results:
        if verbose or r.returncode:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode:
            raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + \
          [obj for obj, _ in results] + ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
