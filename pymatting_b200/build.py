"""Build the sm_100a shared library ``pymatting_b200/_lib/libpmb200.so``.

The library is compiled in-tree with nvcc, one object per translation unit,
and linked with the static CUDA runtime. ``cf_assemble.cu`` is compiled with
``-fmad=false`` so the Laplacian entries follow the reference's IEEE
operation order exactly (no fused multiply-add contraction).
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
TARGET = os.path.join(LIBDIR, "libpmb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-I" + CSRC, "-I" + INCLUDE]
SOURCES = {
    "cf_assemble.cu": ["-fmad=false"],
    "stencil.cu": [],
    "csr.cu": [],
    "lkm.cu": [],
    "foreground.cu": [],
    "foreground_jacobi.cu": [],
    "laplacians.cu": [],
    "knn.cu": [],
    "ichol.cu": ["-fmad=false"],
    "engine.cu": [],
}
HEADERS = ["pm_common.cuh", "stencil.cuh", "csr.cuh", "ichol.cuh"]


def _nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    headers += [os.path.join(INCLUDE, "pymatting_b200.h")]
    objs = []
    relink = force or not os.path.exists(TARGET)
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [_nvcc()] + ARCH + COMMON + extra + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
            relink = True
    if relink or _stale(TARGET, objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-o", TARGET] + objs + ["-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return TARGET


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
