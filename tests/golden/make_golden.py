"""Generate the golden vectors in tests/golden/golden.npz.

The vectors restate the known-answer cases of the reference's own tests
(paths relative to the SHAFFT project):
  * tests/unit/test_fft_partial.cpp:35-40, 231-237 and
    tests/unit/test_fft_partial_fftw.cpp:20-75 -- partial transforms over a
    contiguous block of axes, input v[i] = (sin(0.01 i), cos(0.02 i));
  * tests/unit/test_hipfft_method.cpp:57-163 -- 2x3 Z2Z, input (i+1, 0.25 i);
  * tests/integration/cpp/test_correctness.cpp:145-551 -- delta, plane wave
    exp(+2 pi i k.x / n) with k = (2,3,1) on 8^3 and k = (1,2,0,3,1) on 4^5,
    constant 1.5-0.5i on 8^3, 7-D delta on 4x4x4x4x2x2x2;
  * seeded random inputs on small shapes with prime extents.
Expected outputs are computed here with a naive O(n^2)-per-axis DFT in
float64 whose phases j*k are reduced modulo n in integers before the
sine/cosine (independent of the oracle and of the CUDA code).
Run from the repository root:  python tests/golden/make_golden.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def dft_matrix(n, sign=-1):
    j = np.arange(n)
    m = np.outer(j, j) % n
    return np.exp(sign * 2j * np.pi * m / n)


def naive(x, axes=None, sign=-1):
    x = np.asarray(x, dtype=np.complex128)
    axes = range(x.ndim) if axes is None else axes
    for a in axes:
        x = np.moveaxis(np.tensordot(dft_matrix(x.shape[a], sign), np.moveaxis(x, a, 0), axes=(1, 0)), 0, a)
    return x


def partial_input(n):
    i = np.arange(n, dtype=np.float64)
    return np.sin(0.01 * i) + 1j * np.cos(0.02 * i)


def plane_wave(dims, k):
    grids = np.meshgrid(*[np.arange(d) for d in dims], indexing="ij")
    ph = sum(kk * g / d for kk, g, d in zip(k, grids, dims))
    return np.exp(2j * np.pi * ph)


def main():
    out = {}
    partial = [((2, 3, 4, 5), (0, 1, 2)), ((4, 3, 2, 3, 2), (1, 2, 3)), ((2, 3, 4, 5), (2, 3)),
               ((2, 3, 4, 2), (0, 1, 2, 3)), ((3, 2, 2, 2, 2), (1, 2, 3, 4))]
    for idx, (dims, axes) in enumerate(partial):
        x = partial_input(int(np.prod(dims))).reshape(dims)
        out[f"partial{idx}_in"] = x
        out[f"partial{idx}_axes"] = np.array(axes)
        out[f"partial{idx}_out"] = naive(x, axes)
    x = (np.arange(6) + 1 + 0.25j * np.arange(6)).reshape(2, 3)
    out["axisorder_in"] = x
    out["axisorder_out"] = naive(x)
    d = np.zeros((8, 8, 8), complex)
    d[0, 0, 0] = 1
    out["delta8_in"], out["delta8_out"] = d, naive(d)
    d = np.zeros((8, 8, 8), complex)
    d[3, 1, 6] = 1
    out["delta8s_in"], out["delta8s_out"] = d, naive(d)
    pw = plane_wave((8, 8, 8), (2, 3, 1))
    out["plane8_in"], out["plane8_out"] = pw, naive(pw)
    c = np.full((8, 8, 8), 1.5 - 0.5j)
    out["const8_in"], out["const8_out"] = c, naive(c)
    pw5 = plane_wave((4, 4, 4, 4, 4), (1, 2, 0, 3, 1))
    out["plane5d_in"], out["plane5d_out"] = pw5, naive(pw5)
    d7 = np.zeros((4, 4, 4, 4, 2, 2, 2), complex)
    d7[(0,) * 7] = 1
    out["delta7d_in"], out["delta7d_out"] = d7, naive(d7)
    rng = np.random.Generator(np.random.MT19937(42))
    for name, dims in [("rand_7_11_13", (7, 11, 13)), ("rand_5_6_7", (5, 6, 7)), ("rand_97", (97,)),
                       ("rand_17_19", (17, 19)), ("rand_63_47", (63, 47)), ("rand_3x5x7x3x5", (3, 5, 7, 3, 5))]:
        v = rng.uniform(-1, 1, size=(2,) + dims)
        x = v[0] + 1j * v[1]
        out[f"{name}_in"] = x
        out[f"{name}_out"] = naive(x)
        out[f"{name}_bwd"] = naive(x, sign=+1)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
