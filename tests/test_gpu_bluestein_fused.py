"""Bluestein's element-wise steps fused into the neighbouring specialised
passes (modulate into the first pass's loads, the spectrum multiply and the
demodulate into the last passes' stores): the fused plan has fewer launches,
agrees with the unfused plan (SHAFFT_SM100_BS_FUSE=0) to rounding (the same
operations, contracted into fused multiply-adds differently by the compiler
in the two kernels), forward and backward with the normalisation fused, and
matches the oracle (relative L2 <= 1e-6*log2 N for complex64, 1e-14*log2 N
for complex128)."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

# (dims, precision, launches fused, launches unfused): complex128 plans, the
# convolution FFTs of 1009 (M = 2048, one generic pass) and Bluestein along a
# strided axis keep their element-wise steps
CASES = [((1000003,), 0, 6, 9), ((1000003,), 1, 9, 9), ((100003,), 0, 4, 7), ((4099,), 1, 7, 7),
         ((2, 1009), 0, 6, 6), ((3, 1009), 1, 6, 6), ((5, 100003), 0, 5, 8), ((1009, 3), 0, 6, 6),
         ((100003,), 1, 7, 7)]


def run(dims, prec, x, direction, scale):
    n = x.size
    plan = _sm100.Plan(dims, prec)
    a, b = S.DeviceBuffer(n, prec), S.DeviceBuffer(n, prec)
    a.upload(x)
    plan.execute(a.ptr, b.ptr, direction, scale, 0)
    y = b.download()
    plan.status()
    kinds = [s["kind"] for s in plan.describe()["steps"]]
    plan.destroy()
    return y, kinds


@pytest.mark.parametrize("dims,prec,nf,nu", CASES)
def test_fused_bluestein_bit_identical_and_vs_oracle(monkeypatch, dims, prec, nf, nu):
    n = math.prod(dims)
    x = o.uniform_input(dims, seed=n % 1000, dtype=np.complex128 if prec else np.complex64)
    for direction, sign, scale in ((0, -1, 1.0), (1, 1, 1.0 / n)):
        monkeypatch.setenv("SHAFFT_SM100_BS_FUSE", "1")
        yf, kf = run(dims, prec, x, direction, scale)
        monkeypatch.setenv("SHAFFT_SM100_BS_FUSE", "0")
        yu, ku = run(dims, prec, x, direction, scale)
        assert (len(kf), len(ku)) == (nf, nu), (kf, ku)
        tol = (1e-14 if prec else 1e-6) * math.log2(n)
        assert o.rel_l2(yf, yu) <= tol
        ref = o.fftn(x.astype(np.complex128), sign=sign, precise=bool(prec)).ravel() * scale
        err, err_u = o.rel_l2(yf, ref), o.rel_l2(yu, ref)
        print(f"{dims} prec={prec} dir={direction} fused {err:.3e} unfused {err_u:.3e}")
        assert err <= tol, (dims, direction, err)
