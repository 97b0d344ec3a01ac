"""The C boundary as a C program sees it: tests/c/shafft_c_caller.c is
compiled with gcc against include/shafft/shafft.h and the MPI shim and
linked with libshafft.so; its CPU mode needs no GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "shafft_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("c") / "shafft_c_caller")
    cmd = ["gcc", "-std=c11", "-O1", "-Wall", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "include", "mpi_shim"),
           "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "c", "shafft_c_caller.c"), "-o", exe,
           "-L", LIB, "-lshafft", "-lshafft_mpishim", "-lm", "-Wl,-rpath," + LIB]
    subprocess.run(cmd, check=True)
    return exe


def _run(exe, mode):
    r = subprocess.run([exe, mode], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout
    return r.stdout


def test_c_caller_config_state_errors(caller):
    out = _run(caller, "cpu")
    assert "PASS shafftConfigNDInit" in out and "PASS execute before plan" in out


@pytest.mark.gpu
def test_c_caller_transforms(caller):
    out = _run(caller, "gpu")
    assert "PASS plane wave spectrum" in out and "PASS FFT1D sinusoid spectrum" in out
