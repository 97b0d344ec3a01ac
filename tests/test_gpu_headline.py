"""The headline workloads at full size, checked the way the benchmark runs
them: 512^3 complex64 and 256^3 complex128, input = U[-1,1) noise plus 8
seeded plane waves.

* backward transform against the oracle (the forward one is checked in
  test_gpu_parity.py);
* executeNormalized forward then backward (normalize fused into the last
  pass) returns the input;
* the benchmark's per-kernel launches (shafft_sm100_execute_step with the
  fused normalisation factor) give bit for bit what the reference's call
  sequence gives through the SHAFFT C ABI: execute then normalize
  (src/cpp/shafft_internal.cpp:62-188, the separate normalize kernel of
  src/cpp/fft/hipfft_method/common/normalize.hip:9-77), both directions.

Tolerances (relative L2): 1e-6*log2(N) for complex64, 1e-14*log2(N) for
complex128.
"""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

HEADLINE = [((512, 512, 512), S.C2C), ((256, 256, 256), S.Z2Z)]


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * math.log2(n)


def ok(rc, what=""):
    assert rc == 0, f"{what}: {S.STATUS.get(rc, rc)} {S.last_error_message()}"


def headline_input(dims, prec):
    x = o.uniform_input(dims, seed=42, dtype=np.complex128)
    pw, _ = o.plane_waves(dims, 8, seed=42)
    return (x + pw).astype(np.complex128 if prec == S.Z2Z else np.complex64)


def nd_factor(n, prec):
    """The ND normalisation factor exactly as the library applies it: long
    double 1/sqrt(N), rounded to float for complex64."""
    f = o.nd_norm_factor(n, 1)
    return float(np.float32(f)) if prec == S.C2C else f


class Plan:
    """FFTND through the SHAFFT C ABI with its own two device buffers."""

    def __init__(self, dims, prec):
        self.dims, self.prec = dims, prec
        self.p = S.FFTND()
        ok(self.p.init([1] * len(dims), list(dims), precision=prec), "init")
        ok(self.p.plan(), "plan")
        self.n = self.p.alloc_size()
        self.a = S.DeviceBuffer(self.n, prec)
        self.b = S.DeviceBuffer(self.n, prec)
        ok(self.p.set_buffers(self.a.ptr, self.b.ptr), "setBuffers")

    def load(self, x):
        _, d, _ = self.p.get_buffers()
        (self.a if d == self.a.ptr else self.b).upload(x)

    def result(self):
        _, d, _ = self.p.get_buffers()
        return S.download_ptr(d, self.n, self.prec)

    def close(self):
        self.p.release()
        self.a.free()
        self.b.free()


@pytest.mark.parametrize("dims,prec", HEADLINE)
def test_headline_backward_vs_oracle(dims, prec):
    x = headline_input(dims, prec)
    r = Plan(dims, prec)
    r.load(x)
    ok(r.p.execute(S.BACKWARD), "execute")
    y = r.result()
    r.close()
    ref = o.fftn(x.astype(np.complex128), sign=1, precise=(prec == S.Z2Z)).ravel()
    err = o.rel_l2(y, ref)
    print(f"{dims} prec={prec} backward rel_l2 vs oracle = {err:.3e}")
    assert err <= tol(x.size, prec)


@pytest.mark.parametrize("dims,prec", HEADLINE)
def test_headline_normalized_roundtrip(dims, prec):
    """executeNormalized(FORWARD) then executeNormalized(BACKWARD): the
    transform pair the benchmark times returns the input; the intermediate
    is the forward transform scaled by 1/sqrt(N) (Parseval)."""
    x = headline_input(dims, prec)
    r = Plan(dims, prec)
    r.load(x)
    ok(r.p.execute_normalized(S.FORWARD), "execute")
    y = r.result()
    # unitary scaling keeps the L2 norm
    assert abs(np.linalg.norm(y.astype(np.complex128)) / np.linalg.norm(x.astype(np.complex128)) - 1) \
        <= tol(x.size, prec)
    ok(r.p.execute_normalized(S.BACKWARD), "execute")
    z = r.result()
    r.close()
    err = o.rel_l2(z, x.ravel())
    print(f"{dims} prec={prec} normalized round trip rel_l2 = {err:.3e}")
    assert err <= tol(x.size, prec)


@pytest.mark.parametrize("dims,prec", HEADLINE)
def test_benchmark_launches_match_execute_then_normalize(dims, prec):
    """What the benchmark times -- every kernel of the plan launched with
    shafft_sm100_execute_step and the normalisation fused into the last
    one -- equals execute() + normalize() of the public API bit for bit,
    forward and then backward."""
    torch = pytest.importorskip("torch")
    x = headline_input(dims, prec)
    n = x.size
    f = nd_factor(n, prec)
    # the reference's call sequence through libshafft.so
    r = Plan(dims, prec)
    r.load(x)
    ok(r.p.execute(S.FORWARD), "execute")
    ok(r.p.normalize(), "normalize")
    fwd_ref = r.result()
    ok(r.p.execute(S.BACKWARD), "execute")
    ok(r.p.normalize(), "normalize")
    bwd_ref = r.result()
    r.close()
    # the benchmark's launches
    plan = _sm100.Plan(dims, prec)
    a = S.DeviceBuffer(n, prec)
    b = S.DeviceBuffer(n, prec)
    a.upload(x)
    for i in range(plan.launches):
        plan.execute_step(i, a.ptr, b.ptr, 0, f, 0)
    fwd = b.download()
    for i in range(plan.launches):
        plan.execute_step(i, b.ptr, a.ptr, 1, f, 0)
    bwd = a.download()
    torch.cuda.synchronize()
    plan.destroy()
    np.testing.assert_array_equal(fwd, fwd_ref)
    np.testing.assert_array_equal(bwd, bwd_ref)
    assert o.rel_l2(bwd, x.ravel()) <= tol(n, prec)
