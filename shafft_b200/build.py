"""Build the native libraries of the B200 SHAFFT backend, in tree.

Outputs (shafft_b200/lib/):
  libshafft_sm100.so   sm_100a CUDA kernels + their C ABI (include/shafft_sm100.h)
  libshafft_mpishim.so single-rank MPI (include/mpi_shim/mpi.h) for hosts without MPI
  libshafft.so         SHAFFT C++ API + C ABI (include/shafft/), calls libshafft_sm100

Objects go to shafft_b200/_build/.  Every CUDA source is compiled for
sm_100a only (-gencode arch=compute_100a,code=sm_100a).  Rebuilds only what
is older than its sources.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(PKG, "_build")
INC = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Per-thread default stream: work a caller issues on the NULL stream (plan
# default stream, synchronous copies) goes to the calling thread's own
# stream, so plans driven from different host threads overlap; it still
# synchronises with the legacy default stream other libraries use.
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--default-stream", "per-thread",
                  "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", "-I", INC]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-Wall", "-Wextra", "-Wno-unused-parameter",
            "-I", INC, "-I", os.path.join(INC, "mpi_shim"), "-I", os.path.join(CUDA, "include")]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _headers(d):
    return glob.glob(os.path.join(d, "*.h")) + glob.glob(os.path.join(d, "*.cuh")) + \
        glob.glob(os.path.join(d, "*.hpp"))


def build(verbose: bool = False, jobs: int = 8) -> dict:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    sm = os.path.join(CSRC, "sm100")
    host = os.path.join(CSRC, "host")
    sm_hdrs = _headers(sm) + [os.path.join(INC, "shafft_sm100.h")]
    host_hdrs = (_headers(os.path.join(INC, "shafft")) + _headers(os.path.join(INC, "shafft", "detail"))
                 + [os.path.join(INC, "shafft_sm100.h"), os.path.join(INC, "mpi_shim", "mpi.h")])

    cu_srcs = sorted(glob.glob(os.path.join(sm, "*.cu")))
    jobs_list = []
    objs = []
    for src in cu_srcs:
        o = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(o)
        if _newer(o, [src] + sm_hdrs):
            jobs_list.append([NVCC] + NVFLAGS + ["-c", src, "-o", o])
    shim_src = os.path.join(host, "mpi_shim.cpp")
    shim_o = os.path.join(OBJ, "mpi_shim.o")
    if _newer(shim_o, [shim_src] + host_hdrs):
        jobs_list.append([CXX] + CXXFLAGS + ["-c", shim_src, "-o", shim_o])
    # the C++ API + C ABI, and the Fortran binding's entry points
    host_objs = []
    for name in ("shafft_host", "shafft_f03"):
        src = os.path.join(host, name + ".cpp")
        o = os.path.join(OBJ, name + ".o")
        host_objs.append(o)
        if _newer(o, [src] + host_hdrs):
            jobs_list.append([CXX] + CXXFLAGS + ["-c", src, "-o", o])

    out = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for r in ex.map(_run, jobs_list):
            out.append(r)

    libs = {}
    sm_lib = os.path.join(LIB, "libshafft_sm100.so")
    if _newer(sm_lib, objs):
        out.append(_run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", sm_lib] + objs
                        + ["-cudart", "static"]))
    libs["sm100"] = sm_lib
    shim_lib = os.path.join(LIB, "libshafft_mpishim.so")
    if _newer(shim_lib, [shim_o]):
        out.append(_run([CXX, "-shared", "-o", shim_lib, shim_o]))
    libs["mpishim"] = shim_lib
    host_lib = os.path.join(LIB, "libshafft.so")
    if _newer(host_lib, host_objs + [sm_lib, shim_lib]):
        out.append(_run([CXX, "-shared", "-o", host_lib] + host_objs + ["-L", LIB, "-lshafft_sm100",
                         "-lshafft_mpishim", "-Wl,-rpath,$ORIGIN"]))
    libs["shafft"] = host_lib
    if verbose:
        print("\n".join(x for x in out if x.strip()))
    return libs


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
