"""Build libspeedynn_b200.so in-tree with nvcc for sm_100a.

    python -m speedynn_b200.build          # or speedynn_b200.build.build()

The library is self-contained (static CUDA runtime) and exports only the C ABI
declared in include/speedynn_b200.h.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libspeedynn_b200.so")
SOURCES = ["snn_kernels.cu", "snn_score.cu", "snn_commit.cu", "snn_sorted.cu", "snn_score_tma.cu", "snn_model.cu", "snn_noalloc.cu", "snn_api.cu", "snn_compat.cpp"]
HEADERS = ["snn_internal.h"]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off,-fno-fast-math",
    "--fmad=false",
    "-I" + os.path.join(ROOT, "include"),
]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "speedynn_b200.h"),
                                                                   __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    objs = []
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(HERE, "_build", src + ".o")
        cmd = [nvcc, "-c", os.path.join(CSRC, src), "-o", obj, "-ccbin", "g++"] + NVCC_FLAGS + list(extra)
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-o", tmp, "-ccbin", "g++", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart",
           "static"] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
    print(LIB)
