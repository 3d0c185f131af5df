"""Build libssim2b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python turbo-metrics_b200/build.py        # or: from build import build_library

The kernel translation units are compiled with -fmad=false: every fused
multiply-add in it is written explicitly, so the CPU restatement of the same
arithmetic can reproduce each rounding.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libssim2b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xcompiler", "-ffp-contract=off"]
UNITS = [
    ("ssim2_kernels.cu", ["-fmad=false"]),
    ("ssim2_iir.cu", ["-fmad=false"]),
    ("dssim_kernels.cu", ["-fmad=false"]),
    ("ssim2_engine.cu", []),
    ("ssim2_noalloc.cu", []),
    ("ssim2_server.cu", []),
    ("zensim_kernels.cu", ["-fmad=false"]),
    ("zensim_engine.cu", []),
]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isfile(c) or c == "nvcc"):
            return c
    return "nvcc"


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h", ".inc"))]
    headers.append(os.path.join(HERE, "..", "include", "ssim2b200.h"))
    objs = []
    for src, extra in UNITS:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc()] + ARCH + COMMON + extra + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build_library(verbose=True, force="--force" in sys.argv))
