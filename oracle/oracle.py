"""CPU oracle for the SHAFFT C2C/Z2Z hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker the CUDA path is compared against.  The shipped
library never imports it; only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` do.

It wraps ``oracle/_build/liboracle.so`` (built from ``oracle_fft.c`` by
``oracle/Makefile``), a restatement of the reference's FFTW backend
semantics (src/cpp/fft/fftw_method/fftnd_method.cpp:70-276,
src/cpp/fft/fftw_method/fft1d_method.cpp:130-320): row-major, last axis
fastest, exponent sign -1 forward / +1 backward, unnormalised.  Normalisation
follows src/cpp/shafft_internal.cpp:129-188 (ND: factor (1/sqrt(N))^k computed
in long double) and src/cpp/fft/hipfft_method/fft1d_method.hip:652-679 (1-D:
factor computed from a single-precision sqrt for C2C).

Parity status: pinned.  tests/test_oracle.py checks this oracle against the
reference's known-answer tests (delta, plane wave, constant, Parseval,
naive DFT of the partial-transform unit tests) and against the committed
golden vectors under tests/golden/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-C", _HERE], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(_LIB_PATH)
        i64p = ctypes.POINTER(ctypes.c_int64)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.oracle_fftnd.argtypes = [dp, dp, ctypes.c_int, i64p, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int]
        lib.oracle_fftnd.restype = ctypes.c_int
        lib.oracle_fft_axes.argtypes = [dp, dp, ctypes.c_int, i64p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int]
        lib.oracle_fft_axes.restype = ctypes.c_int
        lib.oracle_naive_dft.argtypes = [dp, dp, ctypes.c_int, i64p, ctypes.c_int]
        lib.oracle_naive_dft.restype = ctypes.c_int
        _lib = lib
    return _lib


def _prep(x):
    x = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    dims = np.asarray(x.shape if x.ndim else (1,), dtype=np.int64)
    return x, dims


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fftn(x, sign: int = -1, precise: bool = False, nthreads: int = 0) -> np.ndarray:
    """Unnormalised C2C DFT over every axis of ``x`` (row-major).

    sign=-1 is SHAFFT/FFTW forward, +1 backward.  precise=True computes in x87
    long double (used as the complex128 oracle), otherwise in float64."""
    x, dims = _prep(x)
    out = np.empty_like(x)
    rc = _load().oracle_fftnd(_dp(x), _dp(out), len(dims),
                              dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                              int(sign), int(bool(precise)), int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle_fftnd failed rc={rc}")
    return out


def fft_axes(x, axes, sign: int = -1, precise: bool = False, nthreads: int = 0):
    """Unnormalised DFT over the listed axes only (partial transform)."""
    x, dims = _prep(x)
    out = np.empty_like(x)
    ax = (ctypes.c_int * max(1, len(axes)))(*axes)
    rc = _load().oracle_fft_axes(_dp(x), _dp(out), len(dims),
                                 dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                 len(axes), ax, int(sign), int(bool(precise)),
                                 int(nthreads))
    if rc != 0:
        raise RuntimeError(f"oracle_fft_axes failed rc={rc}")
    return out


def naive_dft(x, sign: int = -1) -> np.ndarray:
    """O(N^2)-per-axis DFT in long double (restates the reference's naive-DFT
    unit-test oracle, tests/unit/test_fft_partial_fftw.cpp:26-75)."""
    x, dims = _prep(x)
    out = np.empty_like(x)
    rc = _load().oracle_naive_dft(_dp(x), _dp(out), len(dims),
                                  dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                  int(sign))
    if rc != 0:
        raise RuntimeError(f"oracle_naive_dft failed rc={rc}")
    return out


def nd_norm_factor(total: int, exponent: int) -> float:
    """(1/sqrt(N))^k as the reference's ND normalize computes it
    (src/cpp/shafft_internal.cpp:136 with norm_denominator from :329)."""
    den = np.sqrt(np.longdouble(total))
    return float(np.longdouble(1.0) / den ** exponent)


def fft1d_norm_factor(n: int, exponent: int, double: bool) -> float:
    """1-D normalize factor (src/cpp/fft/hipfft_method/fft1d_method.hip:666-671):
    single-precision sqrt for C2C, double for Z2Z."""
    if double:
        return float(1.0 / np.power(np.sqrt(np.float64(n)), exponent))
    return float(np.float32(1.0) / np.power(np.sqrt(np.float32(n)), np.float32(exponent)))


# ---------------------------------------------------------------------------
# Seeded inputs shared by tests and the bench (mt19937_64, seed 42,
# U[-1, 1) drawn re then im per element in row-major order).
# ---------------------------------------------------------------------------

def uniform_input(shape, seed: int = 42, dtype=np.complex64) -> np.ndarray:
    """iid U[-1,1) re/im from numpy's MT19937 stream (the reference's tests
    use std::mt19937_64(42); the exact bit stream differs, the distribution
    and the seeding discipline do not)."""
    rng = np.random.Generator(np.random.MT19937(seed))
    n = int(np.prod(shape))
    v = rng.uniform(-1.0, 1.0, size=2 * n)
    out = (v[0::2] + 1j * v[1::2]).reshape(shape)
    return out.astype(dtype)


def plane_waves(shape, nwaves: int = 8, seed: int = 42):
    """Sum of seeded plane waves a_j * exp(+2 pi i k_j . x / n) with integer
    wavevectors; returns (field, list of (k, a))."""
    rng = np.random.Generator(np.random.MT19937(seed + 1))
    field = np.zeros(shape, dtype=np.complex128)
    waves = []
    for _ in range(nwaves):
        k = tuple(int(rng.integers(0, n)) for n in shape)
        a = float(rng.uniform(0.5, 1.0))
        # separable: prod_d exp(2 pi i k_d x_d / n_d), phases reduced exactly
        term = np.array(a, dtype=np.complex128)
        for ki, n in zip(k, shape):
            e = np.exp(2j * np.pi * ((ki * np.arange(n)) % n) / n)
            term = np.multiply.outer(term, e)
        field += term
        waves.append((k, a))
    return field, waves


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128).ravel()
    b = np.asarray(b, dtype=np.complex128).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def rel_linf(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128).ravel()
    b = np.asarray(b, dtype=np.complex128).ravel()
    den = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0)) if a.size else 0.0
