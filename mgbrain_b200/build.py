"""In-tree build of the CUDA core and the C++ API into
mgbrain_b200/lib/libmgbrain_b200.so (sm_100a only)."""
from __future__ import annotations

import glob
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
OBJ_DIR = os.path.join(ROOT, "_build", "mgbrain_b200")
LIB = os.path.join(LIB_DIR, "libmgbrain_b200.so")
LIB_CHECKED = os.path.join(LIB_DIR, "libmgbrain_b200_checked.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
           "-I" + os.path.join(ROOT, "include")] + ARCH
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-I" + os.path.join(ROOT, "include"),
            "-I/usr/local/cuda/include"]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(verbose=False, checked=False):
    """The library; checked=True builds libmgbrain_b200_checked.so, whose
    kernels test every index they read from memory before using it."""
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = OBJ_DIR + ("_checked" if checked else "")
    lib = LIB_CHECKED if checked else LIB
    os.makedirs(obj_dir, exist_ok=True)
    headers = (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
               + glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True))
    jobs, objs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        if _stale(obj, [src] + headers):
            jobs.append([NVCC] + NVFLAGS + (["-DMGC_CHECKED"] if checked else []) + ["-c", src, "-o", obj])
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp"))):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        if _stale(obj, [src] + headers):
            jobs.append([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    # translation units compile in parallel (the step-kernel instantiations
    # are the long ones)
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        list(pool.map(_run, jobs))
    if _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"])
    if verbose:
        print("built", lib)
    return lib


if __name__ == "__main__":
    import sys
    build(verbose=True, checked="--checked" in sys.argv)
