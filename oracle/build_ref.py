"""Build recipe for the reference's own CPU hot-path ops (test infrastructure).

This script is part of the checker, not of the product.  It compiles the
reference DREAMPlace CPU (OpenMP) operators for the global-placement hot path
straight from their source files under the read-only reference checkout and
writes the resulting Python extension modules into ``oracle/_ref/`` (which is
git-ignored but travels with the repository snapshot to the GPU host, where the
reference checkout does not exist).

Built modules (source files named relative to the reference's ``dreamplace/ops``):

* ``electric_potential_cpp``  - electric_potential/src/electric_density_map.cpp,
  electric_potential/src/electric_force.cpp
* ``dct2_fft2_cpp``           - dct/src/dct2_fft2.cpp
* ``weighted_average_wirelength_cpp_merged`` -
  weighted_average_wirelength/src/weighted_average_wirelength_merged.cpp
* ``pin_pos_cpp``, ``hpwl_cpp``, ``move_boundary_cpp``, ``pws_cpp``,
  ``density_map_cpp``

each linked with utility/src/msg.cpp (the reference's ``utility_cxx``).

Only ``tests/``, ``__graft_entry__`` and ``bench.py``'s CPU-baseline leg load
these modules; nothing in ``dreamplace_b200`` does.

Usage:  python oracle/build_ref.py [--ref PATH] [--jobs 8]
(PATH defaults to $DREAMPLACE_REFERENCE, else /root/reference.)
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

MODULES = {
    "electric_potential_cpp": ["electric_potential/src/electric_density_map.cpp",
                               "electric_potential/src/electric_force.cpp"],
    "dct2_fft2_cpp": ["dct/src/dct2_fft2.cpp"],
    "weighted_average_wirelength_cpp_merged": [
        "weighted_average_wirelength/src/weighted_average_wirelength_merged.cpp"],
    "pin_pos_cpp": ["pin_pos/src/pin_pos.cpp"],
    "hpwl_cpp": ["hpwl/src/hpwl.cpp"],
    "move_boundary_cpp": ["move_boundary/src/move_boundary.cpp"],
    "pws_cpp": ["pin_weight_sum/src/pws.cpp"],
    "density_map_cpp": ["density_map/src/density_map.cpp"],
}


def _torch_flags():
    import torch
    from torch.utils import cpp_extension as ce
    inc = ce.include_paths()
    libdir = os.path.join(os.path.dirname(torch.__file__), "lib")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    major, minor = torch.__version__.split(".")[:2]
    cflags = ["-O3", "-fPIC", "-std=c++17", "-fopenmp",
              f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
              "-DTORCH_API_INCLUDE_EXTENSION_H",
              f"-DTORCH_VERSION_MAJOR={major}", f"-DTORCH_VERSION_MINOR={minor}",
              "-DENABLE_CUDA=0"]
    cflags += ["-I" + p for p in inc]
    cflags += ["-I" + sysconfig.get_paths()["include"]]
    ldflags = ["-shared", "-fopenmp", "-L" + libdir, "-Wl,-rpath," + libdir,
               "-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python"]
    return cflags, ldflags


def build_one(name, srcs, ref, cflags, ldflags, cxx):
    ops = os.path.join(ref, "dreamplace", "ops")
    sources = [os.path.join(ops, s) for s in srcs] + [os.path.join(ops, "utility/src/msg.cpp")]
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    target = os.path.join(OUT, name + ext)
    cmd = [cxx] + cflags + [f"-DTORCH_EXTENSION_NAME={name}", "-I" + ops] + sources + ["-o", target] + ldflags
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building {name} failed:\n{r.stderr[-4000:]}")
    return target


# where the reference checkout is read from: $DREAMPLACE_REFERENCE, else the
# checkout this recipe was written against
DEFAULT_REF = os.environ.get("DREAMPLACE_REFERENCE", "/root/reference")


def available(ref=None):
    return os.path.isdir(os.path.join(ref or DEFAULT_REF, "dreamplace", "ops"))


def build(ref=None, jobs=8, quiet=False):
    ref = ref or DEFAULT_REF
    if not available(ref):
        raise FileNotFoundError(f"reference checkout not found at {ref}")
    os.makedirs(OUT, exist_ok=True)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    cflags, ldflags = _torch_flags()
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = {ex.submit(build_one, n, s, ref, cflags, ldflags, cxx): n for n, s in MODULES.items()}
        for f in cf.as_completed(futs):
            path = f.result()
            if not quiet:
                print("built", os.path.relpath(path, HERE))
    with open(os.path.join(OUT, "__init__.py"), "w") as f:
        f.write("# reference CPU ops built by oracle/build_ref.py (test infrastructure)\n")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--jobs", type=int, default=8)
    a = ap.parse_args()
    build(a.ref, a.jobs)
