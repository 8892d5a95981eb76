"""Builds libswdk.so (the CUDA engine) in-tree for sm_100a with nvcc.

Each source compiles to its own object: the fast-marching file
(swdk_fmst.cu) is built with -fmad=false so its REAL*4 arithmetic keeps the
reference's operation order (no fused multiply-add contraction)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJDIR = os.path.join(HERE, "_build")
HEADER = os.path.join(ROOT, "include", "swdk.h")
# source -> (extra flags, headers it includes)
SOURCES = {
    "swdk.cu": ([], ["swdk_core.cuh", "swdk_eigen.cuh"]),
    "swdk_mlp.cu": ([], []),
    "swdk_fmst.cu": (["-fmad=false"], ["swdk_fmst_march.cuh"]),
    "swdk_lsmr.cu": ([], []),
}
OUT = os.path.join(HERE, "libswdk.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-I" + os.path.join(ROOT, "include"),
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _obj(src):
    return os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(src):
    return [os.path.join(CSRC, src), HEADER] + [os.path.join(CSRC, h) for h in SOURCES[src][1]] + [__file__]


def needs_build():
    return _stale(OUT, [d for s in SOURCES for d in _deps(s)])


def build(verbose=False, force=False):
    if not force and not needs_build():
        return OUT
    os.makedirs(OBJDIR, exist_ok=True)
    objs = []
    for src, (flags, _) in SOURCES.items():
        obj = _obj(src)
        if force or _stale(obj, _deps(src)):
            cmd = [nvcc()] + NVCC_FLAGS + flags + (["-Xptxas", "-v"] if verbose else []) + [
                "-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
            subprocess.run(cmd, check=True)
            os.replace(obj + ".tmp", obj)
        objs.append(obj)
    subprocess.run([nvcc()] + ARCH + ["--shared", "-o", OUT + ".tmp"] + objs, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(OUT)
