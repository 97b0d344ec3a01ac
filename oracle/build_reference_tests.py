"""Compile the reference's own integration test programs, unmodified, against
this repository's SHAFFT headers and libshafft.so -- TEST INFRASTRUCTURE.

The programs are the reference's contract tests of the path this library
replaces (SHAFFT project, tests/integration/cpp/*.cpp and
tests/integration/c/*.c, with tests/include/test_utils.{hpp,h}).  They are
compiled here, where the reference sources lie, straight from those files
(nothing is copied into the repository), with:
  -I include            SHAFFT C/C++ API of this library (shafft.h, shafft.hpp)
  -I include/mpi_shim   single-rank MPI (the image has no MPI)
  -I <reference>/tests/include
  -I <CUDA>/include     (shafft.h names cudaStream_t in its stream setter)
and linked with shafft_b200/lib/libshafft.so and libshafft_mpishim.so.  The
binaries go to oracle/_ref/reftests/ (git-ignored; it travels with the
working tree), where tests/test_gpu_reference_programs.py runs them at one
rank on a GPU.  A program whose sources fail to compile is recorded in
oracle/_ref/reftests/build.json with the compiler's first error lines.

  python oracle/build_reference_tests.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref", "reftests")
LIB = os.path.join(ROOT, "shafft_b200", "lib")
INC = os.path.join(ROOT, "include")


def programs(ref: str):
    cpp = sorted(glob.glob(os.path.join(ref, "tests", "integration", "cpp", "*.cpp")))
    c = sorted(glob.glob(os.path.join(ref, "tests", "integration", "c", "*.c")))
    return cpp + c


def compile_one(src: str, ref: str) -> dict:
    name = os.path.splitext(os.path.basename(src))[0]
    exe = os.path.join(OUT, name)
    is_c = src.endswith(".c")
    cmd = ["gcc" if is_c else "g++", "-O1", "-w",
           "-std=gnu11" if is_c else "-std=c++17",
           "-I", INC, "-I", os.path.join(INC, "mpi_shim"), "-I", os.path.join(ref, "tests", "include"),
           "-I", os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include"),
           src, "-o", exe, "-L", LIB, "-lshafft", "-lshafft_mpishim", "-Wl,-rpath," + LIB,
           "-Wl,-rpath,$ORIGIN/../../../shafft_b200/lib", "-lm"]
    if not is_c:
        cmd.insert(1, "-pthread")
    r = subprocess.run(cmd, capture_output=True, text=True)
    rel = os.path.relpath(src, ref)
    if r.returncode != 0:
        return {"source": rel, "built": False, "error": (r.stdout + r.stderr).splitlines()[:12]}
    return {"source": rel, "built": True, "binary": os.path.relpath(exe, ROOT)}


def build(ref: str = "/root/reference") -> dict:
    if not os.path.isdir(os.path.join(ref, "tests", "integration")):
        return {}
    os.makedirs(OUT, exist_ok=True)
    srcs = programs(ref)
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        res = list(ex.map(lambda s: compile_one(s, ref), srcs))
    summary = {r["source"]: r for r in res}
    with open(os.path.join(OUT, "build.json"), "w") as f:
        json.dump(summary, f, indent=1)
    return summary


if __name__ == "__main__":
    s = build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    for k, v in s.items():
        print(("built   " if v["built"] else "FAILED  ") + k)
        if not v["built"]:
            print("   " + "\n   ".join(v["error"][:6]))
