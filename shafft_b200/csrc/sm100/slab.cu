// Block packing for the slab / pencil exchanges of a distributed N-D transform.
//
// A rank holding a row-major array [outer][n][inner] (n = the axis being
// redistributed) sends peer p the index range [start_p, start_p + len_p) of
// that axis, where (len_p, start_p) is the block partition of n over P parts:
// the first n % P parts get one extra element (the reference's
// block_partition, src/cpp/detail/partition.hpp:40-44).  pack writes the P
// blocks one after the other, each [outer][len_p][inner] row-major, so that
// block p is one contiguous segment of an all-to-all send buffer; unpack is
// the inverse.  Blocks along the outermost axis (outer == 1) are already
// contiguous and need neither.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../../include/shafft_sm100.h"
#include "launch.h"

namespace shafft_sm100 {
namespace {

struct BlockMap {
  int64_t n, q, r;  // n = q * P + r
  __device__ __forceinline__ void locate(int64_t k, int64_t& start, int64_t& len) const {
    // part of column k and that part's (start, len)
    const int64_t big = r * (q + 1);
    int64_t p;
    if (k < big) {
      p = k / (q + 1);
      start = p * (q + 1);
      len = q + 1;
    } else {
      p = r + (k - big) / q;
      start = big + (p - r) * q;
      len = q;
    }
  }
};

// one thread per element of the [outer][n][inner] array; pack: array -> blocks
template <typename C, bool PACK>
__global__ void k_blocks(const C* __restrict__ src, C* __restrict__ dst, int64_t outer, int64_t inner,
                         BlockMap bm) {
  const int64_t row_len = bm.n * inner;
  const int64_t total = outer * row_len;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / row_len, rem = i - row * row_len;
    const int64_t k = rem / inner, ii = rem - k * inner;
    int64_t start, len;
    bm.locate(k, start, len);
    const int64_t b = (outer * start + row * len + (k - start)) * inner + ii;
    if (PACK)
      dst[b] = src[i];
    else
      dst[i] = src[b];
  }
}

template <typename C>
int run_blocks(bool pack, const void* src, void* dst, int64_t outer, int64_t n, int64_t inner,
               int nparts, cudaStream_t s) {
  BlockMap bm{n, n / nparts, n % nparts};
  const int64_t total = outer * n * inner;
  if (total == 0) return 0;
  const int64_t want = (total + 255) / 256;
  const unsigned grid = (unsigned)(want < 148 * 16 ? want : 148 * 16);
  if (pack)
    k_blocks<C, true><<<grid, 256, 0, s>>>(static_cast<const C*>(src), static_cast<C*>(dst), outer, inner, bm);
  else
    k_blocks<C, false><<<grid, 256, 0, s>>>(static_cast<const C*>(src), static_cast<C*>(dst), outer, inner, bm);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : report_error(SHAFFT_SM100_ECUDA, cudaGetErrorString(e));
}

int blocks(bool pack, const void* src, void* dst, int64_t outer, int64_t n, int64_t inner, int nparts,
           int precision, void* stream) {
  if (!src || !dst || src == dst) return report_error(SHAFFT_SM100_EINVAL, "block pack: bad buffers");
  if (outer < 0 || inner < 1 || n < 1 || nparts < 1 || nparts > n || (precision != 0 && precision != 1))
    return report_error(SHAFFT_SM100_EINVAL, "block pack: bad sizes");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return precision ? run_blocks<double2>(pack, src, dst, outer, n, inner, nparts, s)
                   : run_blocks<float2>(pack, src, dst, outer, n, inner, nparts, s);
}

// data[k][c] *= exp(sign * 2 pi i * ((col0 + c) * k mod N) / N), a rows x cols
// array: the twiddle between the two stages of the distributed four-step
// FFT1D (the reference's fft1dTwiddleKernel,
// src/cpp/fft/hipfft_method/1d/fft1d_cooley_tukey_executor.hip:57-83), here
// with the phase reduced exactly in integers before the FP64 sincospi.
template <typename C, typename T>
__global__ void k_twiddle_rows(C* data, int64_t rows, int64_t cols, int64_t col0, int64_t N, int sign) {
  const int64_t total = rows * cols;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i / cols, c = i - k * cols;
    const uint64_t m = ((unsigned __int128)(uint64_t)(col0 + c) * (uint64_t)k) % (uint64_t)N;
    double s, co;
    sincospi((double)sign * 2.0 * ((double)m / (double)N), &s, &co);
    const C a = data[i];
    const T cr = (T)co, sr = (T)s;
    data[i] = C{a.x * cr - a.y * sr, a.x * sr + a.y * cr};
  }
}

int twiddle_rows(void* data, int64_t rows, int64_t cols, int64_t col0, int64_t N, int sign,
                 int precision, void* stream) {
  if (!data || rows < 0 || cols < 0 || col0 < 0 || N < 1 || (sign != 1 && sign != -1) ||
      (precision != 0 && precision != 1))
    return report_error(SHAFFT_SM100_EINVAL, "twiddle: bad arguments");
  const int64_t total = rows * cols;
  if (total == 0) return 0;
  const int64_t want = (total + 255) / 256;
  const unsigned grid = (unsigned)(want < 148 * 16 ? want : 148 * 16);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision)
    k_twiddle_rows<double2, double><<<grid, 256, 0, s>>>(static_cast<double2*>(data), rows, cols, col0, N, sign);
  else
    k_twiddle_rows<float2, float><<<grid, 256, 0, s>>>(static_cast<float2*>(data), rows, cols, col0, N, sign);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : report_error(SHAFFT_SM100_ECUDA, cudaGetErrorString(e));
}

// Distributed Bluestein (the reference's path B for FFT1D lengths not
// divisible by P^2, src/cpp/fft/hipfft_method/1d/fft1d_bluestein_executor.hip):
// each rank holds the M/P-element block of the length-M convolution that
// starts at its N-space offset, so the chirps are generated per block.
//   b[i] = exp(-i pi n^2 / N) at n = n0 + i < N, else 0       (:150-166)
//   v[i] = conj(b[m]) for m < N, conj(b[M - m]) for M - N < m < M,
//          else 0, at m = m0 + i                                 (:168-198)
// with n^2 reduced modulo 2N in integers before the FP64 sincospi, so the
// phase is exact for every N < 2^31.
template <typename C, typename T>
__device__ __forceinline__ C chirp_at(int64_t n, int64_t N, double sign) {
  const uint64_t r = (uint64_t)(((unsigned __int128)(uint64_t)n * (uint64_t)n) % (unsigned __int128)(2 * N));
  double sn, cs;
  sincospi(sign * ((double)r / (double)N), &sn, &cs);
  return C{(T)cs, (T)sn};
}

template <typename C, typename T>
__global__ void k_bluestein_chirps(C* b, C* v, int64_t N, int64_t M, int64_t n0, int64_t m0, int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (b) {
      const int64_t n = n0 + i;
      b[i] = n < N ? chirp_at<C, T>(n, N, -1.0) : C{0, 0};
    }
    if (v) {
      const int64_t m = m0 + i;
      const int64_t j = m < N ? m : (m > M - N && m < M ? M - m : -1);
      v[i] = j >= 0 ? chirp_at<C, T>(j, N, 1.0) : C{0, 0};
    }
  }
}

// dst[i] = conj_out(conj_in(src[i]) * f[i] * scale) for i < valid, 0 for
// valid <= i < count: the modulate, spectrum-multiply and scale+demodulate
// steps of Bluestein (the reference's :38-129 kernels, scale folded in).
template <typename C, typename T>
__global__ void k_chirp_multiply(const C* src, C* dst, const C* f, int64_t count, int64_t valid, int conj_in,
                                 int conj_out, T scale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    C y{0, 0};
    if (i < valid) {
      C a = src[i];
      if (conj_in) a.y = -a.y;
      const C w = f[i];
      y = C{(a.x * w.x - a.y * w.y) * scale, (a.x * w.y + a.y * w.x) * scale};
      if (conj_out) y.y = -y.y;
    }
    dst[i] = y;
  }
}

unsigned ew_blocks(int64_t total) {
  const int64_t want = (total + 255) / 256;
  return (unsigned)(want < 148 * 16 ? want : 148 * 16);
}

int bluestein_chirps(void* b, void* v, int64_t N, int64_t M, int64_t n0, int64_t m0, int64_t count,
                     int precision, void* stream) {
  if ((!b && !v) || N < 1 || M < 2 * N - 1 || n0 < 0 || m0 < 0 || count < 0 ||
      (precision != 0 && precision != 1) || N > ((int64_t)1 << 40))
    return report_error(SHAFFT_SM100_EINVAL, "bluestein chirps: bad arguments");
  if (count == 0) return 0;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision)
    k_bluestein_chirps<double2, double><<<ew_blocks(count), 256, 0, s>>>(
        static_cast<double2*>(b), static_cast<double2*>(v), N, M, n0, m0, count);
  else
    k_bluestein_chirps<float2, float><<<ew_blocks(count), 256, 0, s>>>(
        static_cast<float2*>(b), static_cast<float2*>(v), N, M, n0, m0, count);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : report_error(SHAFFT_SM100_ECUDA, cudaGetErrorString(e));
}

int chirp_multiply(const void* src, void* dst, const void* f, int64_t count, int64_t valid, int conj_in,
                   int conj_out, double scale, int precision, void* stream) {
  if (!src || !dst || !f || count < 0 || valid < 0 || (precision != 0 && precision != 1))
    return report_error(SHAFFT_SM100_EINVAL, "chirp multiply: bad arguments");
  if (count == 0) return 0;
  if (valid > count) valid = count;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision)
    k_chirp_multiply<double2, double><<<ew_blocks(count), 256, 0, s>>>(
        static_cast<const double2*>(src), static_cast<double2*>(dst), static_cast<const double2*>(f), count,
        valid, conj_in, conj_out, scale);
  else
    k_chirp_multiply<float2, float><<<ew_blocks(count), 256, 0, s>>>(
        static_cast<const float2*>(src), static_cast<float2*>(dst), static_cast<const float2*>(f), count,
        valid, conj_in, conj_out, (float)scale);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : report_error(SHAFFT_SM100_ECUDA, cudaGetErrorString(e));
}

}  // namespace
}  // namespace shafft_sm100

extern "C" {

int shafft_sm100_bluestein_chirps(void* b, void* v, int64_t N, int64_t M, int64_t n0, int64_t m0,
                                  int64_t count, int precision, void* stream) {
  return shafft_sm100::bluestein_chirps(b, v, N, M, n0, m0, count, precision, stream);
}

int shafft_sm100_chirp_multiply(const void* src, void* dst, const void* factors, int64_t count,
                                int64_t valid, int conj_in, int conj_out, double scale, int precision,
                                void* stream) {
  return shafft_sm100::chirp_multiply(src, dst, factors, count, valid, conj_in, conj_out, scale,
                                      precision, stream);
}

int shafft_sm100_twiddle_rows(void* data, int64_t rows, int64_t cols, int64_t col0, int64_t N,
                              int sign, int precision, void* stream) {
  return shafft_sm100::twiddle_rows(data, rows, cols, col0, N, sign, precision, stream);
}


int shafft_sm100_pack_blocks(const void* src, void* dst, int64_t outer, int64_t n, int64_t inner,
                             int nparts, int precision, void* stream) {
  return shafft_sm100::blocks(true, src, dst, outer, n, inner, nparts, precision, stream);
}

int shafft_sm100_unpack_blocks(const void* src, void* dst, int64_t outer, int64_t n, int64_t inner,
                               int nparts, int precision, void* stream) {
  return shafft_sm100::blocks(false, src, dst, outer, n, inner, nparts, precision, stream);
}

}  // extern "C"
