"""Builds the CUDA library in-tree: stfwi_b200/libstfwi.so (sm_100a)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libstfwi.so")
SOURCES = [os.path.join(HERE, "csrc", "stfwi.cu"), os.path.join(HERE, "csrc", "nn.cu")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in ("common.cuh", "stencil_parts.cuh", "stencils.cuh", "tma.cuh", "post.cuh", "umma.cuh")] \
    + [os.path.join(ROOT, "include", f) for f in ("stfwi.h", "stfwi_nn.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(verbose: bool = False, force: bool = False, extra=()) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", LIB, *SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else ())
