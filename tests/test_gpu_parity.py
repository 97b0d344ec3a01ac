"""GPU parity of the sm_100a path against the CPU oracle and the golden
vectors, through the SHAFFT C ABI (libshafft.so -> libshafft_sm100.so).

Tolerances (relative L2 against the oracle), the accuracy bar of the path:
  complex64 : 1e-6 * log2(N)
  complex128: 1e-14 * log2(N)
"""
import math

import numpy as np
import pytest

import shafft_b200 as S
from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu


def tol(n, prec):
    return (1e-6 if prec == S.C2C else 1e-14) * max(1.0, math.log2(max(n, 2)))


def ok(rc, what=""):
    assert rc == 0, f"{what}: {S.STATUS.get(rc, rc)} {S.last_error_message()}"


class NDRun:
    """init -> plan -> setBuffers like the reference's tests."""

    def __init__(self, dims, prec=S.C2C, one_d=False):
        self.dims = tuple(dims)
        self.prec = prec
        if one_d:
            self.p = S.FFT1D()
            ok(self.p.init(dims[0], precision=prec), "init")
        else:
            self.p = S.FFTND()
            ok(self.p.init([1] * len(dims), list(dims), precision=prec), "init")
        ok(self.p.plan(), "plan")
        self.n = self.p.alloc_size()
        assert self.n == int(np.prod(dims))
        self.a = S.DeviceBuffer(self.n, prec)
        self.b = S.DeviceBuffer(self.n, prec)
        ok(self.p.set_buffers(self.a.ptr, self.b.ptr), "setBuffers")

    def load(self, x):
        rc, d, _ = self.p.get_buffers()
        ok(rc)
        dt = np.complex128 if self.prec == S.Z2Z else np.complex64
        buf = self.a if d == self.a.ptr else self.b
        buf.upload(np.asarray(x, dtype=dt))

    def result(self):
        rc, d, _ = self.p.get_buffers()
        ok(rc)
        return S.download_ptr(d, self.n, self.prec).reshape(self.dims)


GOLDEN = ["delta8", "delta8s", "plane8", "const8", "plane5d", "delta7d", "rand_7_11_13",
          "rand_5_6_7", "rand_97", "rand_17_19", "rand_63_47", "rand_3x5x7x3x5", "axisorder"]


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("name", GOLDEN)
def test_golden_vectors(golden, name, prec):
    x = golden[f"{name}_in"]
    r = NDRun(x.shape, prec)
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    y = r.result()
    assert o.rel_l2(y, golden[f"{name}_out"]) <= tol(x.size, prec)
    if f"{name}_bwd" in golden:
        r.load(x)
        ok(r.p.execute(S.BACKWARD))
        assert o.rel_l2(r.result(), golden[f"{name}_bwd"]) <= tol(x.size, prec)


SHAPES = [
    (64, 64, 32), (32, 32, 32), (128, 64), (16, 16, 16, 8), (63, 47, 31), (3, 5, 7, 3, 5),
    (2, 3, 2, 3, 2, 3), (2, 2, 3, 2, 2, 3, 2), (3, 2, 2, 2, 3, 2, 2, 2), (1000,), (4096,), (8192,),
    (2048, 2048), (17, 4099), (1, 7, 1), (11, 13), (4096, 3), (625, 81), (343, 49), (1, 1),
    (6000,), (2, 4096, 5),
]


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("dims", SHAPES)
def test_nd_vs_oracle(dims, prec):
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input(dims, seed=11, dtype=dt)
    r = NDRun(dims, prec)
    for direction, sign in ((S.FORWARD, -1), (S.BACKWARD, 1)):
        r.load(x)
        ok(r.p.execute(direction))
        ref = o.fftn(x.astype(np.complex128), sign=sign, precise=(prec == S.Z2Z))
        err = o.rel_l2(r.result(), ref)
        assert err <= tol(x.size, prec), (dims, direction, err)


FFT1D_SIZES = [1, 2, 7, 10, 13, 17, 31, 32, 33, 64, 97, 100, 127, 128, 256, 1000, 1023, 65536, 99991]


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("n", FFT1D_SIZES)
def test_fft1d_vs_oracle(n, prec):
    # sizes of tests/unit/test_FFT1D.cpp:744-780 and test_FFT1D_roundtrip.cpp
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input((n,), seed=n, dtype=dt)
    r = NDRun((n,), prec, one_d=True)
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    ref = o.fftn(x.astype(np.complex128), precise=(prec == S.Z2Z))
    assert o.rel_l2(r.result(), ref) <= tol(n, prec)


@pytest.mark.parametrize("n", [1 << 24, 1488375, 1000003])
@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
def test_fft1d_config_sizes(n, prec):
    """FFT1D at the N = 2^24, 3^5*5^3*7^2 and prime 1,000,003 (Bluestein) sizes."""
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input((n,), seed=3, dtype=dt)
    r = NDRun((n,), prec, one_d=True)
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    ref = o.fftn(x.astype(np.complex128), precise=(prec == S.Z2Z))
    err = o.rel_l2(r.result(), ref)
    print(f"FFT1D N={n} prec={prec} rel_l2={err:.3e}")
    assert err <= tol(n, prec)


@pytest.mark.parametrize("dims", [(64, 64, 32), (32, 32, 32), (128, 64), (16, 16, 16, 8), (63, 47, 31)])
def test_roundtrip_delta(dims):
    """tests/integration/cpp/test_roundtrip.cpp: delta, fwd, normalize, bwd,
    normalize returns the input (tol 1e-4 for C2C)."""
    x = np.zeros(dims, np.complex64)
    x[(0,) * len(dims)] = 1
    r = NDRun(dims)
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    ok(r.p.normalize())
    y = r.result()
    np.testing.assert_allclose(np.abs(y), 1 / math.sqrt(x.size), rtol=1e-4)  # test_delta.cpp
    ok(r.p.execute(S.BACKWARD))
    ok(r.p.normalize())
    np.testing.assert_allclose(r.result(), x, atol=1e-4)


def test_buffer_swap_and_normalize_exponent():
    """After each execute the result is in the buffer getBuffers() calls
    data (test_getbuffers.cpp:60-110); normalize() scales by
    (1/sqrt(N))^k for k executes since the last normalize."""
    dims = (32, 16, 8)
    x = o.uniform_input(dims, dtype=np.complex128)
    r = NDRun(dims, S.Z2Z)
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    rc, d, w = r.p.get_buffers()
    assert (d, w) == (r.b.ptr, r.a.ptr)
    ok(r.p.execute(S.BACKWARD))
    rc, d, w = r.p.get_buffers()
    assert (d, w) == (r.a.ptr, r.b.ptr)
    ok(r.p.normalize())  # k = 2 -> 1/N
    assert o.rel_l2(r.result(), x) < 1e-13
    ok(r.p.normalize())  # k = 0 -> factor 1
    assert o.rel_l2(r.result(), x) < 1e-13


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
@pytest.mark.parametrize("dims", [(64, 64, 32), (63, 47, 31), (1000003,), (4096, 3)])
def test_execute_normalized_matches_execute_then_normalize(dims, prec):
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input(dims, seed=5, dtype=dt)
    r1 = NDRun(dims, prec, one_d=len(dims) == 1)
    r1.load(x)
    ok(r1.p.execute(S.FORWARD))
    ok(r1.p.normalize())
    r2 = NDRun(dims, prec, one_d=len(dims) == 1)
    r2.load(x)
    ok(r2.p.execute_normalized(S.FORWARD))
    np.testing.assert_array_equal(r1.result(), r2.result())


def test_errors_on_gpu_paths():
    p = S.FFTND()
    ok(p.init([1, 1], [8, 8]))
    ok(p.plan())
    assert p.plan() == S.ERR_INVALID_STATE
    assert p.execute(S.FORWARD) == S.ERR_NO_BUFFER
    assert p.normalize() == S.ERR_NO_BUFFER


@pytest.mark.parametrize("prec", [S.C2C, S.Z2Z])
def test_misaligned_buffers_are_refused(prec):
    """The kernel library moves 16-byte vectors: an execute on a buffer that
    is only element-aligned (8 bytes for complex64) or not even that is
    refused with an error before anything is launched, and the context
    stays usable."""
    dims = (64, 64, 32)
    n = math.prod(dims)
    plan = _sm100.Plan(dims, prec, 0)
    a, b = S.DeviceBuffer(n + 2, prec), S.DeviceBuffer(n + 2, prec)
    for off in (8, 4):
        with pytest.raises(_sm100.Sm100Error):
            plan.execute(a.ptr + off, b.ptr, 0, 1.0, 0)
        with pytest.raises(_sm100.Sm100Error):
            plan.execute(a.ptr, b.ptr + off, 0, 1.0, 0)
    x = o.uniform_input(dims, seed=4, dtype=np.complex128 if prec else np.complex64)
    a.upload(x)
    plan.execute(a.ptr, b.ptr, 0, 1.0, 0)
    plan.status()
    ref = o.fftn(x.astype(np.complex128), precise=bool(prec)).ravel()
    assert o.rel_l2(b.download(n), ref) <= (1e-6 if prec == 0 else 1e-14) * math.log2(n)


def test_set_stream():
    torch = pytest.importorskip("torch")
    s = torch.cuda.Stream()
    dims = (64, 32)
    x = o.uniform_input(dims, dtype=np.complex64)
    r = NDRun(dims)
    ok(r.p.set_stream(s.cuda_stream))
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    assert o.rel_l2(r.result(), o.fftn(x.astype(np.complex128))) <= tol(x.size, S.C2C)


@pytest.mark.parametrize("dims,prec", [((512, 512, 512), S.C2C), ((256, 256, 256), S.Z2Z)])
def test_headline_sizes_vs_oracle(dims, prec):
    """512^3 complex64 and 256^3 complex128: input = U[-1,1) noise plus 8
    seeded plane waves; forward vs the oracle (FP64 / long double) and the
    spectral peaks at the plane-wave wavevectors."""
    dt = np.complex128 if prec == S.Z2Z else np.complex64
    x = o.uniform_input(dims, seed=42, dtype=np.complex128)
    pw, waves = o.plane_waves(dims, 8, seed=42)
    x = (x + pw).astype(dt)
    r = NDRun(dims, prec)
    r.load(x)
    ok(r.p.execute(S.FORWARD))
    y = r.result()
    ref = o.fftn(x.astype(np.complex128), precise=(prec == S.Z2Z))
    err = o.rel_l2(y, ref)
    print(f"{dims} prec={prec} rel_l2 vs oracle = {err:.3e} (tol {tol(x.size, prec):.1e})")
    assert err <= tol(x.size, prec)
    n = x.size
    for k, a in waves:
        assert abs(abs(y[k]) - a * n) < 0.01 * a * n


def test_diagnostics_on_stderr():
    """SHAFFT_FFT_DIAG=1 (the reference's switch, src/cpp/fft/common/diag.hpp:17-46)
    prints one tagged line per plan, execute and normalize on stderr."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import shafft_b200 as S\n"
            "p = S.FFTND(); S.check(p.init([1, 1], [32, 16]), 'init'); S.check(p.plan(), 'plan')\n"
            "a = S.DeviceBuffer(512); b = S.DeviceBuffer(512)\n"
            "S.check(p.set_buffers(a.ptr, b.ptr), 'set'); S.check(p.execute(S.FORWARD), 'exec')\n"
            "S.check(p.normalize(), 'norm')\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=root,
                       env=dict(os.environ, SHAFFT_FFT_DIAG="1"), timeout=300)
    assert r.returncode == 0, r.stderr
    err = r.stderr
    assert "[SHAFFT:ND-sm100][r0][fftndPlan] ndim=2 precision=C2C(float) elements=512" in err
    assert "[SHAFFT:ND-sm100][r0][fftndExecute] begin FORWARD" in err
    assert "[SHAFFT:ND-sm100][r0][normalize] exponent=1" in err
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=root,
                       env={k: v for k, v in os.environ.items() if k != "SHAFFT_FFT_DIAG"}, timeout=300)
    assert r.returncode == 0 and "[SHAFFT:" not in r.stderr
