"""Builds the native parts of dreamplace_b200 in-tree.

1. ``libdreamplace_b200.so`` (the C ABI of ``include/dreamplace_b200.h``):
   every ``csrc/*.cu`` compiled by nvcc for sm_100a only
   (``-gencode arch=compute_100a,code=sm_100a``), static CUDA runtime.
2. ``_C*.so``: the PyTorch extension (``csrc/binding.cpp``) linked against the
   library with an ``$ORIGIN`` rpath.

Both land inside the package directory so they travel with the source tree.
Usage: ``python -m dreamplace_b200.build [--force]``.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libdreamplace_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-I" + INCLUDE, "-I" + CSRC]


def ext_path():
    return os.path.join(PKG, "_C" + sysconfig.get_config_var("EXT_SUFFIX"))


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + r.stdout[-3000:] + r.stderr[-6000:])
    return r


def build_library(force=False, jobs=8):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            todo.append((s, o))
    with cf.ThreadPoolExecutor(jobs) as ex:
        list(ex.map(lambda so: _run([NVCC] + NVCC_FLAGS + ["-c", so[0], "-o", so[1]]), todo))
    if force or todo or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", "-soname=libdreamplace_b200.so"])
    return LIB


def build_extension(force=False):
    import torch
    from torch.utils import cpp_extension as ce
    target = ext_path()
    src = os.path.join(CSRC, "binding.cpp")
    if not force and not _newer(target, [src, LIB, os.path.join(INCLUDE, "dreamplace_b200.h")]):
        return target
    torch_lib = os.path.join(os.path.dirname(torch.__file__), "lib")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cuda_inc = "/usr/local/cuda/include"
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-DTORCH_API_INCLUDE_EXTENSION_H", "-DTORCH_EXTENSION_NAME=_C", "-I" + INCLUDE, "-I" + cuda_inc,
           "-I" + sysconfig.get_paths()["include"]]
    cmd += ["-I" + p for p in ce.include_paths()]
    cmd += [src, "-o", target, "-L" + LIBDIR, "-ldreamplace_b200", "-Wl,-rpath,$ORIGIN/lib",
            "-L" + torch_lib, "-Wl,-rpath," + torch_lib, "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu",
            "-ltorch_cuda", "-ltorch_python"]
    _run(cmd)
    return target


def build(force=False, jobs=8):
    build_library(force=force, jobs=jobs)
    return build_extension(force=force)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs))
