"""GPU test of shafft_sm100_bluestein_noalloc, the allocation-free entry point.

Callers that cannot allocate device memory at the point of use -- code that
runs while an allocator lock is held, inside a framework callback that
forbids allocation, or under a device-memory budget reserved up front --
use this entry point: it takes only their input and output buffers and keeps
all of its own state in a static device array.  This file checks, through
the C ABI, that two calls in a row give the same result as the regular
plan-based entry point (shafft_sm100_execute) and as the CPU oracle, within
the tolerance used by the other parity tests, on the legacy default stream
and on a caller's stream, for lengths down to n = 1 and n = 2; and that
sizes beyond its maximum are refused.
It is collected last (file name) so that a stop-at-first-failure run has
already run every other test.
"""
import ctypes
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

MAX_N = 2048


def _entry():
    f = _sm100.load().shafft_sm100_bluestein_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                  ctypes.c_double, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


def _regular(x, prec, direction, scale):
    """The existing entry point: a plan from shafft_sm100_plan_create_nd."""
    n = x.size
    plan = _sm100.Plan((n,), prec)
    a = S.DeviceBuffer(n, prec)
    b = S.DeviceBuffer(n, prec)
    a.upload(x)
    plan.execute(a.ptr, b.ptr, direction, scale, 0)
    y = b.download()  # synchronous copy on the legacy stream the plan ran on
    plan.destroy()
    return y


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
def test_noalloc_matches_regular_entry_point_on_two_calls(prec):
    f = _entry()
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    # two calls in a row, different sizes, directions and scales
    for call, (n, direction, scale) in enumerate([(997, 0, 1.0), (MAX_N, 1, 1.0 / MAX_N)]):
        x = o.uniform_input((n,), seed=100 + call, dtype=dt)
        src = S.DeviceBuffer(n, prec)
        dst = S.DeviceBuffer(n, prec)
        src.upload(x)
        rc = f(ctypes.c_void_p(src.ptr), ctypes.c_void_p(dst.ptr), n, prec, direction, scale, None)
        assert rc == 0, _sm100.load().shafft_sm100_last_error_message()
        y = dst.download()
        ref = _regular(x, prec, direction, scale)
        err = o.rel_l2(y, ref)
        assert err <= _tol(n, prec), (call, n, err)
        err = o.rel_l2(y, _oracle(x, prec, direction, scale))
        assert err <= _tol(n, prec), (call, n, err)


def _oracle(x, prec, direction, scale):
    """The CPU oracle's unnormalised DFT of x (sign -1 forward, +1 backward)
    times scale; long double for complex128."""
    sign = -1 if direction == 0 else 1
    return o.fftn(x.astype(np.complex128), sign=sign, precise=(prec == S.Z2Z)) * scale


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("n", [1, 2, 3, 16, 997, MAX_N])
def test_noalloc_matches_oracle_on_a_caller_stream(prec, n):
    """Two calls in a row on a caller-created stream (not the legacy default
    stream), forward then backward, each against the oracle."""
    torch = pytest.importorskip("torch")
    f = _entry()
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    stream = torch.cuda.Stream()
    for call, (direction, scale) in enumerate([(0, 1.0), (1, 1.0 / n)]):
        x = o.uniform_input((n,), seed=7 * n + call, dtype=dt)
        src = torch.from_numpy(x.copy()).cuda()
        dst = torch.empty_like(src)
        torch.cuda.synchronize()
        rc = f(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), n, prec, direction,
               scale, ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, _sm100.load().shafft_sm100_last_error_message()
        stream.synchronize()
        y = dst.cpu().numpy()
        err = o.rel_l2(y, _oracle(x, prec, direction, scale))
        assert err <= _tol(n, prec), (call, n, err)


def test_noalloc_in_place():
    """in == out is allowed: the input is read into the convolution row
    before the output is written."""
    f = _entry()
    n = 500
    x = o.uniform_input((n,), seed=3, dtype=np.complex64)
    buf = S.DeviceBuffer(n, S.C2C)
    buf.upload(x)
    rc = f(ctypes.c_void_p(buf.ptr), ctypes.c_void_p(buf.ptr), n, S.C2C, 0, 1.0, None)
    assert rc == 0, _sm100.load().shafft_sm100_last_error_message()
    err = o.rel_l2(buf.download(), _oracle(x, S.C2C, 0, 1.0))
    assert err <= _tol(n, S.C2C), err


def test_noalloc_rejects_misaligned_buffers():
    f = _entry()
    n = 1000
    a, b = S.DeviceBuffer(n + 2, S.Z2Z), S.DeviceBuffer(n + 2, S.Z2Z)
    assert f(a.ptr + 8, b.ptr, n, 1, 0, 1.0, None) != 0   # complex128 needs 16 bytes
    assert f(a.ptr + 4, b.ptr, n, 0, 0, 1.0, None) != 0   # complex64 needs 8 bytes
    assert f(a.ptr, b.ptr + 8, n, 0, 0, 1.0, None) == 0   # 8-byte aligned complex64 is fine
    torch = pytest.importorskip("torch")
    torch.cuda.synchronize()


def test_noalloc_rejects_sizes_beyond_maximum():
    f = _entry()
    buf = S.DeviceBuffer(16, S.C2C)
    rc = f(ctypes.c_void_p(buf.ptr), ctypes.c_void_p(buf.ptr), MAX_N + 1, S.C2C, 0, 1.0, None)
    assert rc == 1  # SHAFFT_SM100_EINVAL
    msg = _sm100.load().shafft_sm100_last_error_message().decode()
    assert str(MAX_N) in msg
