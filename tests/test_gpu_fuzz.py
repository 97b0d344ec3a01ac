"""Seeded random shapes against the oracle: 1-4 axes with lengths drawn from
smooth, odd, prime and power-of-two pools, both precisions, forward and
backward with a fused scale, and the tensor-core modes for complex64.  One
test per seed so that a failure names its shape."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

POOLS = {
    "pow2": [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024],
    "smooth": [3, 5, 6, 7, 9, 10, 12, 15, 21, 25, 27, 35, 45, 49, 60, 63, 81, 96, 105, 120, 125, 243, 343],
    "prime": [2, 3, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 97, 101, 127, 131, 211, 257],
}


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


def shape_for(seed):
    rng = np.random.Generator(np.random.MT19937(1000 + seed))
    ndim = int(rng.integers(1, 5))
    dims = []
    for _ in range(ndim):
        pool = POOLS[["pow2", "smooth", "prime"][int(rng.integers(0, 3))]]
        dims.append(int(pool[int(rng.integers(0, len(pool)))]))
    # keep each case small enough for the oracle (<= 2^21 elements)
    while math.prod(dims) > (1 << 21):
        i = int(np.argmax(dims))
        dims[i] = max(1, dims[i] // 4)
    prec = int(rng.integers(0, 2))
    flags = 0
    if prec == 0:
        flags = [0, 0, _sm100.PLAN_TENSOR_CORE, _sm100.PLAN_TC_PRIME_AXES][int(rng.integers(0, 4))]
    return tuple(dims), prec, flags


@pytest.mark.parametrize("seed", range(60))
def test_random_shape_vs_oracle(seed):
    dims, prec, flags = shape_for(seed)
    if flags == _sm100.PLAN_TENSOR_CORE:
        q = _sm100.plan_query(dims, prec, flags)
        if any(s["kind"] != "pass" or not s.get("tc") for s in q["steps"] if s["kind"] != "copy"):
            flags = _sm100.PLAN_TC_PRIME_AXES  # all-tensor-core needs lengths with factors <= 64
    plan = _sm100.Plan(dims, prec, flags)
    dt = np.complex128 if prec else np.complex64
    x = o.uniform_input(dims, seed=seed, dtype=dt)
    n = x.size
    for direction, sign, scale in ((0, -1, 1.0), (1, 1, 1.0 / n)):
        a, b = S.DeviceBuffer(n, prec), S.DeviceBuffer(n, prec)
        a.upload(x)
        plan.execute(a.ptr, b.ptr, direction, scale, 0)
        plan.status()
        y = b.download().reshape(dims)
        ref = o.fftn(x.astype(np.complex128), sign=sign, precise=bool(prec)) * scale
        err = o.rel_l2(y, ref)
        assert err <= tol(n, prec), (dims, prec, flags, direction, err)
