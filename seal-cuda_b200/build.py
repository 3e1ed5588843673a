"""Builds the in-tree shared libraries of the package.

    python seal-cuda_b200/build.py            # libtroy_b200.so (+ pytroy module when present)

* ``lib/libtroy_b200.so``: every ``csrc/*.cu`` compiled by nvcc for sm_100a only
  (``-gencode arch=compute_100a,code=sm_100a -lineinfo``), linked with the CUDA
  runtime. This is the C-ABI library declared in ``include/troy_b200.h``.
* ``lib/pytroy*.so``: the pybind11 module (``binder/pytroy.cpp`` over the C++
  class surface in ``troy/``), linked against libtroy_b200.so.

Objects are cached under ``_build/`` keyed by source mtime; nothing is written
outside the repository.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(ROOT, "_build", "obj")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                  "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
LIBNAME = os.path.join(LIB, "libtroy_b200.so")


def _deps(src):
    hdrs = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return [src] + hdrs


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if not _stale(obj, _deps(src)):
        return obj
    cmd = [NVCC] + NVFLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build_library(verbose=False, jobs=8):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIBNAME, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIBNAME] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIBNAME


def build_pytroy(verbose=False):
    src_dir = os.path.join(HERE, "troy")
    binder = os.path.join(HERE, "binder", "pytroy.cpp")
    if not os.path.exists(binder):
        return None
    import pybind11

    ext = sysconfig.get_config_var("EXT_SUFFIX")
    out = os.path.join(LIB, "pytroy" + ext)
    srcs = [binder] + sorted(glob.glob(os.path.join(src_dir, "*.cpp")))
    deps = srcs + glob.glob(os.path.join(src_dir, "*.hpp")) + [os.path.join(ROOT, "include", "troy_b200.h"), LIBNAME,
                                                                os.path.join(CSRC, "hostmath.hpp")]
    if not _stale(out, deps):
        return out
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
           "-I" + os.path.join(ROOT, "include"), "-I" + src_dir, "-I" + CSRC, "-I/usr/local/cuda/include"] + srcs + \
          ["-o", out, "-L" + LIB, "-ltroy_b200", "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64", "-lcudart"]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"pytroy build failed:\n{r.stdout}\n{r.stderr}")
    return out


def main():
    verbose = "-v" in sys.argv
    print(build_library(verbose))
    p = build_pytroy(verbose)
    if p:
        print(p)


if __name__ == "__main__":
    main()
