"""Build libsbp_b200.so in-tree with nvcc for sm_100a (B200): one object per source under
_build/ (compiled in parallel), then one shared library."""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["sbp_kernels.cu", "sbp_sparse.cu", "sbp_sort.cu", "sbp_engine.cu", "sbp_mlp.cu", "sbp_learned.cu",
           "sbp_batched.cu", "sbp_noalloc.cu", "sbp_ingest.cu", "sbp_evaluate.cu",
           "sbp_eval_small.cu"]
HEADERS = ["sbp_device.cuh", "sbp_kernels.cuh", "sbp_sort.cuh", "sbp_engine.cuh", "sbp_mlp.cuh", "sbp_steps.cuh",
           "sbp_error.h",
           os.path.join("..", "..", "include", "sbp_b200.h")]
LIB = os.path.join(HERE, "libsbp_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]
# The batched persistent kernel reads blockmodel state that other CTAs of the same launch
# update: its global loads go to L2 (cache-global), never a possibly stale L1 line.
FILE_FLAGS = {"sbp_batched.cu": ["-Xptxas", "-dlcm=cg"]}


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
    os.makedirs(OBJ, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        cmd = [nvcc] + NVCC_FLAGS + FILE_FLAGS.get(src, []) + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
