"""Measured planning (SHAFFT_SM100_PLAN_MEASURE): the plan chosen by timing
the candidates on the GPU is correct, its choice is cached per shape, and a
second plan of the same shape reuses the cached choice."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


@pytest.mark.parametrize("dims,prec,flags", [((1488375,), 0, 0), ((121500,), 1, 0),
                                             ((4096, 61), 0, _sm100.PLAN_TC_PRIME_AXES),
                                             ((1 << 20,), 0, 0)])
def test_measured_plan_parity_and_cache(tmp_path, monkeypatch, dims, prec, flags):
    cache = tmp_path / "plans.txt"
    monkeypatch.setenv("SHAFFT_SM100_PLAN_CACHE", str(cache))
    plan = _sm100.Plan(dims, prec, flags | _sm100.PLAN_MEASURE)
    lines = cache.read_text().splitlines() if cache.exists() else []
    q = _sm100.plan_query(dims, prec, flags | _sm100.PLAN_MEASURE)
    assert [s["L"] for s in q["steps"]] == [s["L"] for s in plan.describe()["steps"]]
    dt = np.complex128 if prec else np.complex64
    x = o.uniform_input(dims, seed=5, dtype=dt)
    a, b = S.DeviceBuffer(x.size, prec), S.DeviceBuffer(x.size, prec)
    a.upload(x)
    plan.execute(a.ptr, b.ptr, 0, 1.0, 0)
    plan.status()
    y = b.download().reshape(dims)
    assert o.rel_l2(y, o.fftn(x.astype(np.complex128), precise=bool(prec))) <= tol(x.size, prec)
    _sm100.Plan(dims, prec, flags | _sm100.PLAN_MEASURE)   # cache hit: nothing appended
    after = cache.read_text().splitlines() if cache.exists() else []
    assert after == lines
    assert len(lines) <= 1
