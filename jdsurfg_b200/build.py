"""Builds libswdk.so (the CUDA engine) in-tree for sm_100a with nvcc."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(HERE, "csrc", f) for f in ("swdk.cu", "swdk_mlp.cu")]
DEPS = [os.path.join(HERE, "csrc", f) for f in ("swdk.cu", "swdk_mlp.cu", "swdk_core.cuh", "swdk_eigen.cuh")] + [
    os.path.join(ROOT, "include", "swdk.h")]
OUT = os.path.join(HERE, "libswdk.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--shared", "-Xcompiler", "-fPIC",
    "-I" + os.path.join(ROOT, "include"),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(verbose=False, force=False):
    if not force and not needs_build():
        return OUT
    cmd = [nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + SRC + ["-o", OUT + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(OUT)
