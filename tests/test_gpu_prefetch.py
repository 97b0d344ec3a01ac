"""The complex64 512-point specialised pass with an L2 prefetch of a later
tile (k_fft_fast_pf; on by default for row-input passes, one wave ahead)
against the plain kernel (SHAFFT_SM100_PREFETCH_ROW=0): the prefetch only
warms L2, the butterflies are the same, so the outputs must be
bit-identical.  A third run also prefetches the column-input passes
(SHAFFT_SM100_PREFETCH_COL=4); a fourth loads the column-input passes with
256-byte L2 fetches instead (SHAFFT_SM100_COL_FETCH=256); a fifth issues the
row prefetches one 128-byte line at a time instead of as one bulk
asynchronous prefetch per row (SHAFFT_SM100_BULK_PREFETCH=0).  The
switches are read once per process, so each setting runs in a child
process.  Every result is also checked against the oracle (1e-6*log2(N)).  The shapes cover the transposing pair of a 3-D
plan with few and many tiles (the prefetch target past the last tile is
skipped), a row pass followed by other lengths, and the four-step twiddled
row pass of a 1-D plan."""
import math
import os
import subprocess
import sys

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [(16, 512, 512), (3, 512, 512), (512, 64, 512), (1 << 18,), (40, 512, 512)]


def run_all(out_dir):
    """Forward and scaled backward of every case; results saved as .npy,
    with each plan's description (which steps prefetch)."""
    for i, dims in enumerate(CASES):
        plan = _sm100.Plan(dims, S.C2C, 0)
        x = o.uniform_input(dims, seed=300 + i, dtype=np.complex64)
        n = x.size
        for direction, scale in ((0, 1.0), (1, 1.0 / n)):
            a, b = S.DeviceBuffer(n, S.C2C), S.DeviceBuffer(n, S.C2C)
            a.upload(x)
            plan.execute(a.ptr, b.ptr, direction, scale, 0)
            plan.status()
            np.save(os.path.join(out_dir, f"c{i}_d{direction}.npy"), b.download())
        pf = [s.get("prefetch", 0) for s in plan.describe()["steps"]]
        np.save(os.path.join(out_dir, f"c{i}_pf.npy"), np.array(pf))
        plan.destroy()


CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import test_gpu_prefetch as t
t.run_all(sys.argv[2])
"""


def _child(tmp_path, name, **env):
    d = tmp_path / name
    d.mkdir()
    switches = ("SHAFFT_SM100_PREFETCH", "SHAFFT_SM100_BULK_PREFETCH", "SHAFFT_SM100_COL_FETCH")
    e = {k: v for k, v in os.environ.items() if not k.startswith(switches)}
    e.update(env)
    script = tmp_path / "child.py"
    script.write_text(CHILD)
    r = subprocess.run([sys.executable, str(script), ROOT, str(d)], env=e, timeout=600)
    assert r.returncode == 0
    return d


def test_prefetching_pass_matches_plain_pass_bitwise(tmp_path):
    on = _child(tmp_path, "on")
    off = _child(tmp_path, "off", SHAFFT_SM100_PREFETCH_ROW="0")
    col = _child(tmp_path, "col", SHAFFT_SM100_PREFETCH_COL="4")
    fetch = _child(tmp_path, "fetch", SHAFFT_SM100_COL_FETCH="256")
    lines = _child(tmp_path, "lines", SHAFFT_SM100_BULK_PREFETCH="0")
    for i, dims in enumerate(CASES):
        # the default prefetches every 512-point row pass, and only those
        pf_on, pf_off, pf_col = (np.load(d / f"c{i}_pf.npy") for d in (on, off, col))
        assert pf_on.max() == 4 and not pf_off.any(), (dims, pf_on, pf_off)
        assert (pf_col >= pf_on).all()
        x = o.uniform_input(dims, seed=300 + i, dtype=np.complex64)
        n = x.size
        tol = 1e-6 * max(1.0, math.log2(n))
        ref = o.fftn(x.astype(np.complex128)).ravel()
        for direction in (0, 1):
            y_on = np.load(on / f"c{i}_d{direction}.npy")
            y_off = np.load(off / f"c{i}_d{direction}.npy")
            y_col = np.load(col / f"c{i}_d{direction}.npy")
            assert np.array_equal(y_on.view(np.uint32), y_off.view(np.uint32)), (dims, direction)
            assert np.array_equal(y_col.view(np.uint32), y_off.view(np.uint32)), (dims, direction)
            y_fetch = np.load(fetch / f"c{i}_d{direction}.npy")
            assert np.array_equal(y_fetch.view(np.uint32), y_off.view(np.uint32)), (dims, direction)
            y_lines = np.load(lines / f"c{i}_d{direction}.npy")
            assert np.array_equal(y_lines.view(np.uint32), y_off.view(np.uint32)), (dims, direction)
            if direction == 0:
                assert o.rel_l2(y_on, ref) <= tol, dims
            else:
                assert o.rel_l2(y_on, o.fftn(x.astype(np.complex128), sign=1).ravel() / n) <= tol, dims
