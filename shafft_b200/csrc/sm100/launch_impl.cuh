// Definitions of Launch<T> (see launch.h); included by launch_f32.cu and
// launch_f64.cu only.
#pragma once
#include <algorithm>

#include "kernels.cuh"
#include "launch.h"

namespace shafft_sm100 {

static inline unsigned ew_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

template <typename T>
cudaError_t Launch<T>::init() {
  return cudaFuncSetAttribute(k_fft_pass<T, 0, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              200 * 1024);
}

template <typename T>
cudaError_t Launch<T>::pass(const PassGeom& g, const C* in, C* out, const PassTables<C>& tb,
                            size_t smem, cudaStream_t s) {
  const int64_t grid = std::min<int64_t>(g.ntiles, 148 * 64);
  k_fft_pass<T, 0, 0><<<(unsigned)grid, kThreads, smem, s>>>(g, in, out, tb);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::scale_copy(const C* src, C* dst, int64_t n, T factor, int conj,
                                  cudaStream_t s) {
  k_scale_copy<T><<<ew_grid(n), 256, 0, s>>>(src, dst, n, factor, conj);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::bs_modulate(const C* src, C* dst, int64_t L, int64_t M, int64_t I,
                                   int64_t total, const C* chirp, int conj, cudaStream_t s) {
  k_bs_modulate<T><<<ew_grid(total), 256, 0, s>>>(src, dst, L, M, I, total, chirp, conj);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::bs_mulh(C* d, const C* H, int64_t M, int64_t total, cudaStream_t s) {
  k_bs_mulh<T><<<ew_grid(total), 256, 0, s>>>(d, H, M, total);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::bs_demod(const C* src, C* dst, int64_t L, int64_t M, int64_t I, int64_t total,
                                const C* chirp, int conj, T scale, cudaStream_t s) {
  k_bs_demod<T><<<ew_grid(total), 256, 0, s>>>(src, dst, L, M, I, total, chirp, conj, scale);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::gen_twiddle(C* out, int64_t count, int64_t mult, int64_t N, cudaStream_t s) {
  k_gen_twiddle<T><<<ew_grid(count), 256, 0, s>>>(out, count, mult, N);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::gen_chirp(C* out, int64_t L, cudaStream_t s) {
  k_gen_chirp<T><<<ew_grid(L), 256, 0, s>>>(out, L);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::gen_bs_kernel(C* h, const C* chirp, int64_t L, int64_t M, cudaStream_t s) {
  k_gen_bs_kernel<T><<<ew_grid(M), 256, 0, s>>>(h, chirp, L, M);
  return cudaGetLastError();
}

}  // namespace shafft_sm100
