"""The cluster plane pass (k_fft_plane_cluster): both axes of each 512 x 512
complex64 plane in one HBM pass, a 16-CTA thread-block cluster exchanging
the plane through distributed shared memory.  Checked against the CPU oracle
(relative L2 <= 1e-6*log2 N) on stacks of planes smaller and larger than
the number of clusters the GPU holds at once, in place and out of place,
forward and backward with the normalisation fused."""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu


def tol(n):
    return 1e-6 * math.log2(n)


@pytest.fixture
def cluster_on(monkeypatch):
    monkeypatch.setenv("SHAFFT_SM100_PLANE_CLUSTER", "1")


@pytest.mark.parametrize("dims", [(512, 512), (3, 512, 512), (20, 512, 512), (2, 3, 512, 512)])
def test_cluster_plane_vs_oracle(cluster_on, dims):
    plan = _sm100.Plan(dims, 0)
    steps = plan.describe()["steps"]
    assert steps[0]["kind"] == "plane" and steps[0].get("cluster") == 16, steps
    n = math.prod(dims)
    x = o.uniform_input(dims, seed=17, dtype=np.complex64)
    a, b = S.DeviceBuffer(n), S.DeviceBuffer(n)
    for direction, sign, scale in ((0, -1, 1.0), (1, 1, 1.0 / n)):
        a.upload(x)
        plan.execute(a.ptr, b.ptr, direction, scale, 0)
        y = b.download().reshape(dims)
        plan.status()
        ref = o.fftn(x.astype(np.complex128), sign=sign) * scale
        err = o.rel_l2(y, ref)
        print(f"{dims} dir={direction} rel_l2={err:.3e}")
        assert err <= tol(n), (dims, direction, err)
    plan.destroy()


def test_cluster_plane_through_the_api_roundtrip(cluster_on):
    """FFTND through the SHAFFT C ABI (execute, normalize, execute,
    normalize) on 4 x 512 x 512 returns the input; the forward transform
    matches the oracle."""
    dims = (4, 512, 512)
    n = math.prod(dims)
    x = o.uniform_input(dims, seed=5, dtype=np.complex64)
    p = S.FFTND()
    assert p.init([1, 1, 1], list(dims)) == 0 and p.plan() == 0
    a, b = S.DeviceBuffer(n), S.DeviceBuffer(n)
    assert p.set_buffers(a.ptr, b.ptr) == 0
    a.upload(x)
    assert p.execute(S.FORWARD) == 0
    _, d, _ = p.get_buffers()
    y = S.download_ptr(d, n, S.C2C).reshape(dims)
    assert o.rel_l2(y, o.fftn(x.astype(np.complex128))) <= tol(n)
    assert p.normalize() == 0
    assert p.execute(S.BACKWARD) == 0 and p.normalize() == 0
    _, d, _ = p.get_buffers()
    assert o.rel_l2(S.download_ptr(d, n, S.C2C).reshape(dims), x) <= tol(n)
    p.release()


def test_cluster_plane_off_keeps_two_passes(monkeypatch):
    monkeypatch.setenv("SHAFFT_SM100_PLANE_CLUSTER", "0")
    steps = _sm100.plan_query((4, 512, 512), 0)["steps"]
    assert all(s["kind"] == "pass" for s in steps)
