"""Column passes of length 256 and 512 fed by bulk tensor copies
(k_fft_fast_tma, opt-in with SHAFFT_SM100_TMA=1, so run in a child process
since the switch is read once) against the default register-load kernel:
the same butterflies in the same order, so the outputs must be bit-identical.
Both are also checked against the oracle (1e-6*log2(N) C2C, 1e-14*log2(N)
Z2Z).  The shapes cover one-, two- and outer-batch column views, in-place
and out-of-place passes, and fused four-step twiddles."""
import json
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

CASES = [((512, 32, 64), 0), ((512, 32, 64), 1), ((256, 40, 48), 0), ((256, 48, 40), 1), ((1 << 18,), 1),
         ((1 << 16,), 0), ((1 << 17,), 0), ((1 << 21,), 1), ((2, 256, 8, 256), 0), ((512, 512), 0)]


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


def run_all(out_dir):
    """Forward and scaled backward of every case; results saved as .npy."""
    for i, (dims, prec) in enumerate(CASES):
        plan = _sm100.Plan(dims, prec, 0)
        dt = np.complex128 if prec else np.complex64
        x = o.uniform_input(dims, seed=100 + i, dtype=dt)
        n = x.size
        for direction, scale in ((0, 1.0), (1, 1.0 / n)):
            a, b = S.DeviceBuffer(n, prec), S.DeviceBuffer(n, prec)
            a.upload(x)
            plan.execute(a.ptr, b.ptr, direction, scale, 0)
            plan.status()
            np.save(os.path.join(out_dir, f"c{i}_d{direction}.npy"), b.download())


CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import test_gpu_tma as t
t.run_all(sys.argv[2])
assert t._sm100.tma_launch_count() > 0  # switched on: the bulk-copy kernel ran
"""


def test_plans_take_tma_eligible_column_passes():
    for dims, prec in CASES:
        q = _sm100.plan_query(dims, prec, 0)
        assert any(s["kind"] == "pass" and s.get("fast") and not s["in_row"] and s["L"] in (256, 512)
                   for s in q["steps"]), (dims, q)


def test_tma_matches_register_load_kernel_bitwise(tmp_path):
    on, off = tmp_path / "on", tmp_path / "off"
    on.mkdir()
    off.mkdir()
    if os.environ.get("SHAFFT_SM100_TMA", "0") != "0":
        pytest.skip("this process must run the default register-load kernel")
    before = _sm100.tma_launch_count()
    run_all(str(off))
    assert _sm100.tma_launch_count() == before  # default: register-load kernel only
    env = dict(os.environ, SHAFFT_SM100_TMA="1")
    script = tmp_path / "child.py"
    script.write_text(CHILD)
    r = subprocess.run([sys.executable, str(script), ROOT, str(on)], env=env, timeout=600)
    assert r.returncode == 0
    for i, (dims, prec) in enumerate(CASES):
        dt = np.complex128 if prec else np.complex64
        x = o.uniform_input(dims, seed=100 + i, dtype=dt)
        n = x.size
        for direction, sign, scale in ((0, -1, 1.0), (1, 1, 1.0 / n)):
            y_on = np.load(on / f"c{i}_d{direction}.npy")
            y_off = np.load(off / f"c{i}_d{direction}.npy")
            assert np.array_equal(y_on.view(np.uint8), y_off.view(np.uint8)), (dims, prec, direction)
            ref = o.fftn(x.astype(np.complex128), sign=sign, precise=bool(prec)) * scale
            err = o.rel_l2(y_on.reshape(dims), ref)
            assert err <= tol(n, prec), (dims, prec, direction, err)
