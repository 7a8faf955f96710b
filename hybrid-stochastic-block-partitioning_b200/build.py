"""Build libsbp_b200.so in-tree with nvcc for sm_100a (B200)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["sbp_kernels.cu", "sbp_sparse.cu", "sbp_sort.cu", "sbp_engine.cu", "sbp_mlp.cu", "sbp_learned.cu",
           "sbp_noalloc.cu"]
HEADERS = ["sbp_device.cuh", "sbp_kernels.cuh", "sbp_sort.cuh", "sbp_engine.cuh", "sbp_mlp.cuh", os.path.join("..", "..", "include", "sbp_b200.h")]
LIB = os.path.join(HERE, "libsbp_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.abspath(__file__)]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
