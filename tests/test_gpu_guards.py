"""Guard bytes around device allocations (SHAFFT_SM100_CANARY=1), a safety
net for out-of-bounds writes: every kind of pass the planner builds runs on
guarded user buffers and guarded plan tables / scratch, and no guard byte
may change; a write planted on the host just outside a buffer (an ordinary
in-bounds copy into the guard area, no kernel involved) must be reported by
shafft_sm100_check_guards and by the free of that buffer.  Runs in child
processes because the switch is read once per process."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CLEAN = r'''
import ctypes, math, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import shafft_b200 as S
from shafft_b200 import _sm100
from oracle import oracle as o
lib = _sm100.load()
cases = [((64, 64, 32), 0, 0), ((512, 512, 8), 0, 0), ((63, 47, 31), 0, 0), ((1 << 20,), 0, 0),
         ((1488375,), 0, 0), ((1000003,), 0, 0), ((100003,), 1, 0), ((256, 256, 16), 1, 0),
         ((4096, 61), 0, _sm100.PLAN_TC_PRIME_AXES), ((16, 64, 64), 0, _sm100.PLAN_TENSOR_CORE),
         ((7, 11, 13), 1, 0), ((1,), 0, 0), ((2, 3), 1, 0)]
for dims, prec, flags in cases:
    n = math.prod(dims)
    x = o.uniform_input(dims, seed=1, dtype=np.complex128 if prec else np.complex64)
    p = _sm100.Plan(dims, prec, flags)
    a, b = S.DeviceBuffer(n, prec), S.DeviceBuffer(n, prec)
    for direction in (0, 1):
        a.upload(x)
        p.execute(a.ptr, b.ptr, direction, 1.0 / n if direction else 1.0, 0)
        p.status()
    y = b.download()
    assert lib.shafft_sm100_check_guards() == 0, (dims, lib.shafft_sm100_last_error_message())
    ref = o.fftn(x.astype(np.complex128), sign=1, precise=bool(prec)).ravel() / n
    assert o.rel_l2(y, ref) <= (1e-14 if prec else 1e-6) * max(1, math.log2(max(n, 2))), dims
    assert lib.shafft_sm100_plan_destroy(p.handle) == 0, lib.shafft_sm100_last_error_message()
    p.handle = None
    a.free(); b.free()
print("CLEAN_OK")
'''

PLANTED = r'''
import ctypes, sys
sys.path.insert(0, sys.argv[1])
import shafft_b200 as S
from shafft_b200 import _sm100
lib = _sm100.load()
side = sys.argv[2]
p = ctypes.c_void_p()
assert lib.shafft_sm100_malloc(ctypes.byref(p), 800) == 0
assert lib.shafft_sm100_check_guards() == 0
junk = (ctypes.c_ubyte * 16)(*range(16))
target = p.value + 800 if side == "after" else p.value - 16
assert lib.shafft_sm100_memcpy(ctypes.c_void_p(target), junk, 16, 1, None) == 0
rc = lib.shafft_sm100_check_guards()
msg = lib.shafft_sm100_last_error_message().decode()
assert rc == 3 and side in msg and "out-of-bounds write" in msg, (rc, msg)
rc = lib.shafft_sm100_free(p)
assert rc == 3, rc
print("PLANTED_OK", msg)
'''


def _run(code, *args):
    env = dict(os.environ, SHAFFT_SM100_CANARY="1")
    return subprocess.run([sys.executable, "-c", code, ROOT, *args], capture_output=True, text=True,
                          env=env, timeout=600, cwd=ROOT)


def test_no_pass_writes_outside_its_buffers():
    r = _run(CLEAN)
    assert r.returncode == 0 and "CLEAN_OK" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("side", ["after", "before"])
def test_planted_write_outside_a_buffer_is_reported(side):
    r = _run(PLANTED, side)
    assert r.returncode == 0 and "PLANTED_OK" in r.stdout, r.stdout + r.stderr
