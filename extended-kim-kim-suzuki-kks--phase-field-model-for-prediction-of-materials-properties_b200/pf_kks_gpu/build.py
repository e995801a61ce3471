"""Build the sm_100a shared library ``libkks_b200.so`` in-tree.

Each CUDA source is compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a``
into an object file under ``csrc/_build/``, and the objects are linked into
``pf_kks_gpu/libkks_b200.so`` against cuFFT. ``kks_scalar.cu`` (the single-thread
prologue / decide kernels) and ``kks_init.cu`` (initial state) are compiled
with ``-fmad=false`` so that their arithmetic keeps numpy's float64 rounding;
the field kernels keep FMA contraction.

``--bounds-check`` builds the debug variant ``pf_kks_gpu/libkks_b200_check.so``
(objects under ``csrc/_build_check/``) with ``-DKKS_BOUNDS_CHECK``: the fused
passes check each block's ranges and record the first failure instead of
faulting (csrc/kks_check.cuh, kks_bounds_report); load it with
``KKS_LIBRARY=<path>``.

Usage: python -m pf_kks_gpu.build [--force] [--verbose] [--bounds-check]
"""

import argparse
import os
import shutil
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(ROOT_DIR, "csrc")
REPO_DIR = os.path.dirname(ROOT_DIR)
INCLUDE = os.path.join(REPO_DIR, "include")
BUILD_DIR = os.path.join(CSRC, "_build")
LIB_NAME = "libkks_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)
CHECK_BUILD_DIR = os.path.join(CSRC, "_build_check")
CHECK_LIB_PATH = os.path.join(PKG_DIR, "libkks_b200_check.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = {
    "kks_scalar.cu": ["-fmad=false"],
    "kks_fields.cu": [],
    "kks_abi.cu": [],
    "kks_fft.cu": [],
    "kks_fft64.cu": [],
    "kks_noalloc.cu": [],
    "kks_adjoint.cu": [],
    "kks_init.cu": ["-fmad=false"],
}


def cuda_home():
    for cand in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if cand and os.path.exists(os.path.join(cand, "bin", "nvcc")):
            return cand
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found (set CUDA_HOME)")


def _deps(src):
    """Sources plus the headers they include."""
    return [src, os.path.join(CSRC, "kks_internal.cuh"), os.path.join(CSRC, "kks_fft.cuh"),
            os.path.join(CSRC, "kks_check.cuh"), os.path.join(CSRC, "kks_pointwise.cuh"), os.path.join(INCLUDE, "kks.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra_flags=(), bounds_check=False):
    """Compile the CUDA sources and link the shared library; returns its path.
    ``bounds_check``: the -DKKS_BOUNDS_CHECK debug variant (its own objects
    and library file)."""
    home = cuda_home()
    nvcc = os.path.join(home, "bin", "nvcc")
    build_dir, lib_path = (CHECK_BUILD_DIR, CHECK_LIB_PATH) if bounds_check else (BUILD_DIR, LIB_PATH)
    if bounds_check:
        extra_flags = (*extra_flags, "-DKKS_BOUNDS_CHECK")
    os.makedirs(build_dir, exist_ok=True)
    objs = []
    for src, flags in SOURCES.items():
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, _deps(path)):
            cmd = [nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
                   *flags, *extra_flags, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if force or _stale(lib_path, objs):
        lib_dir = os.path.join(home, "lib64")
        cmd = [nvcc, *ARCH, "-shared", "-o", lib_path, *objs, "-L", lib_dir, "-lcufft",
               "-Xlinker", "-rpath=" + lib_dir]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return lib_path


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--bounds-check", action="store_true", help="build the -DKKS_BOUNDS_CHECK debug variant")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, bounds_check=a.bounds_check))
