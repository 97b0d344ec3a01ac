"""Pin the CPU oracle (oracle/oracle_fft.c) against the reference's
known-answer tests and the committed golden vectors.  CPU only."""
import numpy as np
import pytest

from oracle import oracle as o

PARTIAL = 5


def test_golden_partial_transforms(golden):
    # tests/unit/test_fft_partial_fftw.cpp:26-75 (tol 1e-10 there)
    for i in range(PARTIAL):
        x = golden[f"partial{i}_in"]
        axes = [int(a) for a in golden[f"partial{i}_axes"]]
        y = o.fft_axes(x, axes)
        assert o.rel_linf(y, golden[f"partial{i}_out"]) < 1e-12


def test_golden_axis_order(golden):
    # tests/unit/test_hipfft_method.cpp:57-163: 2x3 Z2Z, input (i+1, 0.25 i)
    y = o.fftn(golden["axisorder_in"])
    assert o.rel_linf(y, golden["axisorder_out"]) < 1e-13


@pytest.mark.parametrize("name", ["delta8", "delta8s", "plane8", "const8", "plane5d", "delta7d",
                                  "rand_7_11_13", "rand_5_6_7", "rand_97", "rand_17_19",
                                  "rand_63_47", "rand_3x5x7x3x5"])
@pytest.mark.parametrize("precise", [False, True])
def test_golden_full(golden, name, precise):
    y = o.fftn(golden[f"{name}_in"], precise=precise)
    assert o.rel_l2(y, golden[f"{name}_out"]) < 1e-13
    if f"{name}_bwd" in golden:
        yb = o.fftn(golden[f"{name}_in"], sign=1, precise=precise)
        assert o.rel_l2(yb, golden[f"{name}_bwd"]) < 1e-13


def test_known_answers_analytic():
    # tests/integration/cpp/test_correctness.cpp:145-344
    d = np.zeros((8, 8, 8), complex)
    d[0, 0, 0] = 1
    np.testing.assert_allclose(o.fftn(d), np.ones((8, 8, 8)), atol=1e-12)
    g = np.meshgrid(*[np.arange(8)] * 3, indexing="ij")
    pw = np.exp(2j * np.pi * (2 * g[0] + 3 * g[1] + 1 * g[2]) / 8)
    y = o.fftn(pw)
    expect = np.zeros((8, 8, 8), complex)
    expect[2, 3, 1] = 512
    np.testing.assert_allclose(y, expect, atol=1e-9)
    c = np.full((8, 8, 8), 1.5 - 0.5j)
    y = o.fftn(c)
    assert abs(y[0, 0, 0] - (1.5 - 0.5j) * 512) < 1e-9
    y[0, 0, 0] = 0
    assert np.max(np.abs(y)) < 1e-9


def test_parseval_and_roundtrip():
    # test_correctness.cpp:349-421 (Parseval 16x16x8) and test_roundtrip.cpp
    x = o.uniform_input((16, 16, 8), dtype=np.complex128)
    y = o.fftn(x)
    n = x.size
    assert abs(np.sum(np.abs(x) ** 2) - np.sum(np.abs(y) ** 2) / n) < 1e-10 * np.sum(np.abs(x) ** 2)
    for shape in [(64, 64, 32), (63, 47, 31), (16, 16, 16, 8), (128, 64)]:
        x = o.uniform_input(shape, seed=7, dtype=np.complex128)
        f = o.nd_norm_factor(x.size, 1)
        z = o.fftn(o.fftn(x) * f, sign=1) * f
        assert o.rel_l2(z, x) < 1e-13


@pytest.mark.parametrize("n", [1, 2, 7, 10, 13, 17, 31, 64, 97, 100, 127, 256, 1000, 1023, 4099])
def test_1d_sizes_vs_numpy(n):
    # tests/unit/test_FFT1D.cpp:744-780 sizes and a few primes (Bluestein path)
    x = o.uniform_input((n,), seed=n, dtype=np.complex128)
    assert o.rel_l2(o.fftn(x), np.fft.fft(x)) < 1e-13
    assert o.rel_l2(o.fftn(x, precise=True), np.fft.fft(x)) < 1e-13
    assert o.rel_l2(o.fftn(x, sign=1), np.fft.ifft(x) * n) < 1e-13


def test_long_double_beats_double():
    x = o.uniform_input((1 << 12,), dtype=np.complex128)
    ref = o.naive_dft(x)
    e64 = o.rel_l2(o.fftn(x), ref)
    eld = o.rel_l2(o.fftn(x, precise=True), ref)
    assert eld <= e64 * 1.01 and eld < 1e-15


def test_norm_factors_follow_reference():
    # ND: long double sqrt (shafft_internal.cpp:136); 1-D C2C: float sqrt (fft1d_method.hip:667)
    assert o.nd_norm_factor(512 ** 3, 1) == pytest.approx(1 / np.sqrt(512.0 ** 3), rel=1e-15)
    assert o.fft1d_norm_factor(1000003, 1, double=False) == float(np.float32(1) / np.sqrt(np.float32(1000003)))
    assert o.nd_norm_factor(100, 0) == 1.0


@pytest.mark.parametrize("dims", [(2, 3, 2, 2, 3, 2, 2, 2), (2,) * 9, (3, 2, 2, 2, 2, 2, 2, 2, 2, 2),
                                  (2,) * 11, (2,) * 12])
def test_high_rank_tensors_vs_naive_dft(dims):
    """8-D to 12-D tensors against the naive DFT, as the reference's
    high-dimensional unit tests do (tests/unit/test_fft_highdim.cpp:186-205):
    the oracle's FFT and its naive DFT agree to FP64 rounding, forward and
    backward."""
    x = o.uniform_input(dims, seed=len(dims), dtype=np.complex128)
    for sign in (-1, 1):
        y = o.fftn(x, sign=sign)
        ref = o.naive_dft(x, sign=sign)
        assert o.rel_l2(y, ref) <= 1e-13, (dims, sign)
