/*
 * oracle_fft.c -- CPU oracle for the SHAFFT C2C/Z2Z hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; nothing in the shipped library links, loads or calls it.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * What it restates (reference paths are relative to the SHAFFT project):
 *   - src/cpp/fft/fftw_method/fftnd_method.cpp:34-66, 70-234, 236-276
 *       one multi-dimensional C2C DFT over the whole row-major tensor
 *       (last axis fastest), FFTW_FORWARD = -1 in the exponent, no scaling.
 *       The oracle plans out-of-place (the reference's in-place plan that is
 *       executed out of place is not reproduced).
 *   - src/cpp/fft/fftw_method/fft1d_method.cpp:130-320
 *       the 1-D transform of length N, same sign and scaling convention.
 *   - src/cpp/fft/fftw_method/common/normalize.cpp:6-32 and
 *     src/cpp/shafft_internal.cpp:129-188
 *       normalisation is a separate real multiply by (1/sqrt(N))^k; it is
 *       left to the caller of this oracle (tests apply it in float64).
 *
 * FFTW itself (a third-party dependency of the reference, not vendored, not
 * installed here) computes the same mathematical DFT; this file restates the
 * textbook algorithms instead:
 *   - Stockham auto-sort mixed-radix decimation in time.  For a stage of
 *     radix p after sub-transforms of length l (l' = l*p):
 *         A'[s][k + l*q] = sum_r w_p^{r q} * ( w_{l'}^{r k} * A[s + (n/l') r][k] )
 *     where A[s][k] is the length-l DFT of the decimated sequence
 *     x[s + (n/l) j].  Radix-p butterflies are direct O(p^2) sums.
 *   - Bluestein's chirp-z identity for lengths with a prime factor > 61:
 *         nk = (n^2 + k^2 - (k-n)^2)/2,
 *         X[k] = c[k] sum_n (x[n] c[n]) conj(c[k-n]),  c[m] = exp(sign*i*pi*m^2/N)
 *     evaluated as a cyclic convolution of power-of-two length M >= 2N-1,
 *     with m^2 reduced modulo 2N in integer arithmetic before the sine/cosine.
 *
 * Two arithmetic types are built from the same source: double (the FP64
 * oracle used for complex64 parity) and x87 long double (64-bit mantissa,
 * used for the complex128 parity so that errors near 1e-14 are resolvable).
 * Inputs and outputs are always interleaved float64 (re, im) pairs.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAX_FACTORS 64
#define ORACLE_DIRECT_PRIME_MAX 61

/* ------------------------------------------------------------------------ */
/* Generic body, instantiated for double and long double.                    */
/* ------------------------------------------------------------------------ */

#define REAL double
#define SUFFIX _d
#define COS cos
#define SIN sin
#define PI_R 3.14159265358979323846264338327950288
#include "oracle_fft_body.h"
#undef REAL
#undef SUFFIX
#undef COS
#undef SIN
#undef PI_R

#define REAL long double
#define SUFFIX _ld
#define COS cosl
#define SIN sinl
#define PI_R 3.14159265358979323846264338327950288L
#include "oracle_fft_body.h"
#undef REAL
#undef SUFFIX
#undef COS
#undef SIN
#undef PI_R

/* ------------------------------------------------------------------------ */
/* Exported C ABI                                                            */
/* ------------------------------------------------------------------------ */

/* Multi-dimensional C2C DFT of a row-major tensor.
 *   in, out : interleaved (re, im) float64, prod(dims) complex elements;
 *             in == out is allowed.
 *   sign    : -1 forward (FFTW_FORWARD), +1 backward.  Unnormalised.
 *   precise : 0 -> FP64 arithmetic, 1 -> x87 long double arithmetic.
 *   nthreads: OpenMP threads over independent lines (<=0: library default).
 * Returns 0 on success, -1 on a bad argument, -2 on allocation failure. */
int oracle_fftnd(const double* in, double* out, int ndim, const int64_t* dims,
                 int sign, int precise, int nthreads) {
  if (!in || !out || !dims || ndim < 1 || (sign != 1 && sign != -1)) return -1;
  for (int a = 0; a < ndim; ++a)
    if (dims[a] < 1) return -1;
  if (precise) return fftnd_ld(in, out, ndim, dims, sign, nthreads);
  return fftnd_d(in, out, ndim, dims, sign, nthreads);
}

/* Transform only the listed axes (a partial multi-dimensional DFT); used to
 * restate the reference's partial-transform unit tests. */
int oracle_fft_axes(const double* in, double* out, int ndim, const int64_t* dims,
                    int naxes, const int* axes, int sign, int precise, int nthreads) {
  if (!in || !out || !dims || ndim < 1 || naxes < 0 || (naxes && !axes) ||
      (sign != 1 && sign != -1))
    return -1;
  for (int a = 0; a < ndim; ++a)
    if (dims[a] < 1) return -1;
  for (int i = 0; i < naxes; ++i)
    if (axes[i] < 0 || axes[i] >= ndim) return -1;
  if (precise) return fftaxes_ld(in, out, ndim, dims, naxes, axes, sign, nthreads);
  return fftaxes_d(in, out, ndim, dims, naxes, axes, sign, nthreads);
}

/* Naive O(N^2) DFT over all axes of a small tensor, evaluated separably one
 * axis at a time in long double with exactly reduced phases.  This is the
 * restatement of the reference's naive-DFT unit-test oracle
 * (tests/unit/test_fft_partial_fftw.cpp:26-75). */
int oracle_naive_dft(const double* in, double* out, int ndim, const int64_t* dims,
                     int sign) {
  if (!in || !out || !dims || ndim < 1 || (sign != 1 && sign != -1)) return -1;
  return naive_ld(in, out, ndim, dims, sign);
}

/* out[i] *= factor for n complex elements (float64). */
void oracle_scale(double* data, int64_t n, double factor) {
  for (int64_t i = 0; i < 2 * n; ++i) data[i] *= factor;
}
