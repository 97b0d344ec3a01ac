"""The reference's own integration test programs, unmodified, run at one MPI
rank against this library on the GPU.

oracle/build_reference_tests.py compiles the SHAFFT project's
tests/integration/cpp/*.cpp and tests/integration/c/*.c (with
tests/include/test_utils.{hpp,h}) against include/shafft/ and
libshafft.so, into oracle/_ref/reftests/ -- only where the reference sources
are present, so on a machine without them this module skips.  Each program
prints one PASS/FAIL line per case (its own tolerances: test_utils.hpp
check_rel_error with TOL_F = 1e-5, TOL_D = 1e-12 scaled by sqrt(log N)).

Expected differences, each a documented behaviour change of this backend:
  test_c_api "shafftGetBackendName": the program accepts only "FFTW" or
      "hipFFT"; this backend reports "sm100".
Every other case of every program must pass.  Cases that need more than one
rank are skipped by the programs themselves at one rank (they report PASS).
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "reftests")

PROGRAMS = [
    "test_FFT1D_roundtrip", "test_axes", "test_backend", "test_configuration_modes",
    "test_correctness", "test_delta", "test_double", "test_errors", "test_getbuffers",
    "test_highdim", "test_inactive_ranks", "test_initcart", "test_layout", "test_roundtrip",
    "test_c_FFT1D", "test_c_api", "test_c_roundtrip",
]

EXPECTED_FAILURES = {"test_c_api": {"shafftGetBackendName"}}

CASE = re.compile(r"^\s+(\S.*?)\s+(PASS|FAIL)\b(.*)$")


def cases(stdout: str):
    out = {}
    for line in stdout.splitlines():
        m = CASE.match(line)
        if m:
            out[m.group(1).strip()] = (m.group(2), m.group(3).strip())
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", PROGRAMS)
def test_reference_program(name):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{name} not built: the reference sources were absent when "
                    "oracle/build_reference_tests.py last ran")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, cwd=ROOT)
    res = cases(r.stdout)
    print(r.stdout)
    assert res, f"{name}: no PASS/FAIL lines (rc={r.returncode})\n{r.stdout}\n{r.stderr}"
    failed = {k for k, (v, _) in res.items() if v == "FAIL"}
    expected = EXPECTED_FAILURES.get(name, set())
    assert failed == expected, (f"{name}: unexpected results {sorted(failed ^ expected)}\n"
                                f"{r.stdout}\n{r.stderr[-2000:]}")
    if not expected:
        assert r.returncode == 0, f"{name}: rc={r.returncode}\n{r.stderr[-2000:]}"
