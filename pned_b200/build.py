"""Builds libpned_gpu.so in-tree for sm_100a (nvcc; no JIT cache).

The library is the product: CUDA kernels plus the C ABI declared in
include/pned_gpu.h.  It is written next to this file so that it travels with
the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpned_gpu.so")
SOURCES = ["host_model.cpp", "host_io.cpp", "device.cu", "hv_staged.cu", "hv_qtile.cu", "hv_sector.cu", "krylov.cu", "slots.cu"]
HEADERS = ["pned_internal.h", "kernels.cuh", "device.cuh", os.path.join("..", "..", "include", "pned_gpu.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS + [os.path.basename(__file__)]:
        path = os.path.join(CSRC, f) if f != os.path.basename(__file__) else __file__
        if os.path.getmtime(path) > t:
            return True
    return False


def build(force: bool = False, verbose: bool = False, sanitize: str = "") -> str:
    """Compile every CUDA/C++ source into pned_b200/libpned_gpu.so.

    sanitize ("address" or "undefined") instruments the host-only sources
    (model compiler, planners, file formats) with that gcc sanitizer, for the
    CPU tests; an address-sanitized library needs libasan preloaded
    (LD_PRELOAD=$(gcc -print-file-name=libasan.so), ASAN_OPTIONS=detect_leaks=0).
    Rebuild without it (force=True) afterwards."""
    if sanitize not in ("", "address", "undefined"):
        raise ValueError("sanitize: 'address' or 'undefined'")
    if not force and not _stale():
        return LIB
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp", "-lineinfo", "-ccbin", "g++",
              "-I" + os.path.join(ROOT, "include")]
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        cmd = [nvcc, *common, *ARCH, "-c", os.path.join(CSRC, src), "-o", obj]
        if sanitize and src.endswith(".cpp"):
            cmd += ["-Xcompiler", f"-fsanitize={sanitize},-fno-omit-frame-pointer,-g"]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", *ARCH, "-o", tmp, *objs, "-Xcompiler", "-fopenmp", "-lcudart"]
    if sanitize:
        cmd += ["-Xcompiler", f"-fsanitize={sanitize}"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    san = next((a.split("=", 1)[1] for a in sys.argv if a.startswith("--sanitize=")), "")
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, sanitize=san)
    print(LIB)
