"""Build recipe of the sm_100a shared library ``libcbm_b200.so``.

The library holds the CUDA kernels, the host orchestration and the C ABI
declared in ``include/cbm_b200.h``.  It is built in the package directory so
that it travels with the source tree; ``python cerebellum_simulation_b200/build.py``
rebuilds it (run as a file: importing the package needs the library).
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libcbm_b200.so")
BUILD_DIR = os.path.join(PKG, "_build")

# -fmad=false: every float/double operation of the step is rounded once, in
# source order, like the CPU reference built without FP contraction.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I", os.path.join(ROOT, "include"),
]

SOURCES = ["cbm_state.cpp", "cbm_netgen.cpp", "cbm_sim.cu", "cbm_kernels.cu", "cbm_pass_vec.cu", "cbm_capi.cu", "cbm_noalloc.cu",
           "cbm_mlp.cu"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libcbm_b200.so")
    return path


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(verbose=False, force=False):
    """Compile every source for sm_100a and link libcbm_b200.so."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "cbm_b200.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc()] + NVCC_FLAGS + ["-c", path, "-o", obj]
            if src.endswith(".cpp"):
                cmd = [nvcc()] + NVCC_FLAGS + ["-x", "c++", "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build_library(verbose=True, force="--force" in sys.argv)
    print(LIB)
