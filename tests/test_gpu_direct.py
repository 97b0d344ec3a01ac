"""Axes with a prime factor above 13 transformed by the direct-DFT pass
(outputs evaluated in symmetric pairs) up to the planner's limit, and by
Bluestein beyond it: forward and normalised backward against the oracle,
both precisions, along contiguous and strided axes.  Tolerances as in the
other parity tests: 1e-6*log2(N) for complex64, 1e-14*log2(N) for
complex128."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

# (dims, expect a direct pass for every non-smooth axis)
CASES = [((263,), True), ((4, 331), True), ((211, 17, 3), True), ((2, 353), True), ((139, 139), True),
         ((34, 5), True), ((2 * 181,), True), ((367,), False), ((3, 509), False)]


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("dims,direct", CASES)
def test_direct_and_bluestein_axes_vs_oracle(dims, direct, prec):
    n = math.prod(dims)
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input(dims, seed=n % 1000, dtype=dt)
    plan = _sm100.Plan(dims, prec)
    kinds = [s["kind"] for s in plan.describe()["steps"]]
    assert ("bluestein_modulate" not in kinds) == direct, kinds
    a, b = S.DeviceBuffer(n, prec), S.DeviceBuffer(n, prec)
    a.upload(x)
    plan.execute(a.ptr, b.ptr, 0, 1.0, 0)
    y = b.download().reshape(dims)
    ref = o.fftn(x.astype(np.complex128), precise=(prec == S.Z2Z))
    assert o.rel_l2(y, ref) <= tol(n, prec), ("forward", o.rel_l2(y, ref))
    # backward with the normalisation fused returns the input
    a.upload(y)
    plan.execute(a.ptr, b.ptr, 1, 1.0 / n, 0)
    z = b.download().reshape(dims)
    assert o.rel_l2(z, x) <= 2 * tol(n, prec), ("round trip", o.rel_l2(z, x))
    plan.status()
    plan.destroy()
