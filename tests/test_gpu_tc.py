"""Tensor-core form (SHAFFT_SM100_PLAN_TENSOR_CORE): complex64 plans whose
passes are tcgen05 split-FP16 DFT GEMMs, checked against the CPU oracle at
the complex64 tolerance 1e-6 * log2(N) (relative L2)."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

TC = _sm100.PLAN_TENSOR_CORE


def tol(n):
    return 1e-6 * max(1.0, math.log2(max(n, 2)))


def run(plan, x, direction=0, scale=1.0):
    n = x.size
    a = S.DeviceBuffer(n)
    b = S.DeviceBuffer(n)
    a.upload(np.ascontiguousarray(x, dtype=np.complex64))
    plan.execute(a.ptr, b.ptr, direction, scale, 0)
    plan.status()
    return b.download().reshape(x.shape)


SHAPES = [(64,), (61,), (16,), (48,), (2,), (4096,), (1000,), (1 << 16,), (64, 64, 32), (7, 11, 13),
          (128, 256), (35, 27, 45), (3, 64, 5), (2048, 33)]


@pytest.mark.parametrize("dims", SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_tc_forward_backward_vs_oracle(dims):
    q = _sm100.plan_query(dims, 0, TC)
    assert all(s.get("tc") == 1 for s in q["steps"] if s["kind"] == "pass"), q
    plan = _sm100.Plan(dims, 0, TC)
    x = o.uniform_input(dims, seed=42, dtype=np.complex64)
    n = x.size
    y = run(plan, x)
    ref = o.fftn(x.astype(np.complex128))
    assert o.rel_l2(y, ref) <= tol(n), o.rel_l2(y, ref)
    yb = run(plan, x, direction=1, scale=1.0 / n)
    refb = o.fftn(x.astype(np.complex128), sign=1) / n
    assert o.rel_l2(yb, refb) <= tol(n), o.rel_l2(yb, refb)


@pytest.mark.parametrize("n", [1 << 20, 1488375, 1 << 24])
def test_tc_fft1d_config_sizes(n):
    """FFT1D sizes of the tensor-core configuration (2^24, 3^5*5^3*7^2)."""
    plan = _sm100.Plan((n,), 0, TC)
    x = o.uniform_input((n,), seed=42, dtype=np.complex64)
    y = run(plan, x)
    ref = o.fftn(x.astype(np.complex128))
    assert o.rel_l2(y, ref) <= tol(n), o.rel_l2(y, ref)


def test_tc_bluestein_prime():
    n = 1000003
    q = _sm100.plan_query((n,), 0, TC)
    assert any(s["kind"] == "bluestein_modulate" for s in q["steps"])
    plan = _sm100.Plan((n,), 0, TC)
    x = o.uniform_input((n,), seed=42, dtype=np.complex64)
    y = run(plan, x)
    ref = o.fftn(x.astype(np.complex128))
    assert o.rel_l2(y, ref) <= tol(n), o.rel_l2(y, ref)


def test_tc_wide_dynamic_range():
    """Rows whose entries span many binades (a spike over noise) keep the
    split-precision error bound: each row is scaled by its own maximum."""
    dims = (64, 64)
    rng = np.random.Generator(np.random.MT19937(7))
    x = (rng.uniform(-1, 1, dims) + 1j * rng.uniform(-1, 1, dims)) * 1e-3
    x[5, 7] = 3e4
    x[40, :] *= 1e-6
    x = x.astype(np.complex64)
    plan = _sm100.Plan(dims, 0, TC)
    y = run(plan, x)
    ref = o.fftn(x.astype(np.complex128))
    assert o.rel_l2(y, ref) <= tol(x.size)


def test_tc_every_length_2_to_64():
    """One tensor-core pass for every length 2..64 (primes included), batched
    along a second axis so that tiles hold full 128-row groups."""
    for L in range(2, 65):
        dims = (300, L)
        plan = _sm100.Plan(dims, 0, TC)
        x = o.uniform_input(dims, seed=L, dtype=np.complex64)
        y = run(plan, x)
        ref = o.fftn(x.astype(np.complex128))
        assert o.rel_l2(y, ref) <= tol(x.size), L


PRIME_SHAPES = [(4096, 61), (61, 61, 61), (53, 59, 61), (512, 61, 16), (17, 19, 23, 8), (8, 1024, 47),
                (61 * 64 * 32,)]


@pytest.mark.parametrize("dims", PRIME_SHAPES, ids=lambda d: "x".join(map(str, d)))
def test_tc_prime_axes_hybrid_vs_oracle(dims):
    """Hybrid mode: tensor-core passes on the axes with a prime factor above
    13, plain passes elsewhere; both directions against the oracle."""
    PRIME = _sm100.PLAN_TC_PRIME_AXES
    q = _sm100.plan_query(dims, 0, PRIME)
    assert any(s.get("tc") for s in q["steps"]), q
    plan = _sm100.Plan(dims, 0, PRIME)
    x = o.uniform_input(dims, seed=11, dtype=np.complex64)
    n = x.size
    y = run(plan, x)
    ref = o.fftn(x.astype(np.complex128))
    assert o.rel_l2(y, ref) <= tol(n), o.rel_l2(y, ref)
    yb = run(plan, x, direction=1, scale=1.0 / n)
    refb = o.fftn(x.astype(np.complex128), sign=1) / n
    assert o.rel_l2(yb, refb) <= tol(n), o.rel_l2(yb, refb)
