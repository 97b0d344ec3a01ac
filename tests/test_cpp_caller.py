"""The C++ API as a C++ program sees it: tests/cpp/shafft_cpp_caller.cpp is
compiled with g++ against include/shafft/shafft.hpp and linked with
libshafft.so; it checks host-side behaviour only (no GPU)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "shafft_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "shafft_cpp_caller")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "include", "mpi_shim"),
           "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "shafft_cpp_caller.cpp"), "-o", exe,
           "-L", LIB, "-lshafft", "-lshafft_mpishim", "-Wl,-rpath," + LIB]
    subprocess.run(cmd, check=True)
    return exe


def test_cpp_caller_host_behaviour(caller):
    r = subprocess.run([caller], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout
    assert "PASS moved-from plan is uninitialised" in r.stdout
