// Definitions of Launch<T> (see launch.h); included by launch_f32.cu and
// launch_f64.cu only.
#pragma once
#include <algorithm>

#include "fast.cuh"
#include "kernels.cuh"
#include "launch.h"

namespace shafft_sm100 {

static inline unsigned ew_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

// Compile-time radix plans of the specialised passes: (L, R0, R1, R2, threads).
// Every stage gives each thread a whole number of 16-byte-chunk butterflies.
template <typename T>
struct FastTable;
#define SHAFFT_FAST_LIST_F32(X) \
  X(16, 4, 4, 1, 32)            \
  X(32, 8, 4, 1, 32)            \
  X(64, 8, 8, 1, 64)            \
  X(128, 8, 4, 4, 128)          \
  X(256, 8, 8, 4, 256)          \
  X(512, 8, 8, 8, 256)          \
  X(1024, 8, 8, 16, 512)
#define SHAFFT_FAST_LIST_F64(X) \
  X(16, 4, 4, 1, 32)            \
  X(32, 8, 4, 1, 32)            \
  X(64, 8, 8, 1, 64)            \
  X(128, 8, 4, 4, 128)          \
  X(256, 8, 8, 4, 128)          \
  X(512, 8, 8, 8, 256)


#define SHAFFT_PLANE_LIST_F32(X) \
  X(128, 8, 4, 4, 128)           \
  X(256, 8, 8, 4, 256)           \
  X(512, 8, 8, 8, 256)           \
  X(1024, 8, 8, 16, 512)
#define SHAFFT_PLANE_LIST_F64(X) \
  X(128, 8, 4, 4, 128)           \
  X(256, 8, 8, 4, 128)           \
  X(512, 8, 8, 8, 256)

template <typename KernelT, typename... Args>
static cudaError_t launch_cluster(KernelT kernel, int planes, int cluster, int threads, size_t smem,
                                  cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(planes * cluster), 1, 1);
  cfg.blockDim = dim3((unsigned)threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename T>
static cudaError_t fast_attr_all();

#ifdef SHAFFT_INSTANTIATE_F32
template <>
cudaError_t fast_attr_all<float>() {
  cudaError_t e = cudaSuccess;
#define SHAFFT_ATTR(L, A, B, C_, NT)                                                             \
  if (e == cudaSuccess)                                                                          \
    e = cudaFuncSetAttribute(k_fft_fast<float, L, A, B, C_, NT, false>,                          \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);              \
  if (e == cudaSuccess)                                                                          \
    e = cudaFuncSetAttribute(k_fft_fast<float, L, A, B, C_, NT, true>,                           \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
  SHAFFT_FAST_LIST_F32(SHAFFT_ATTR)
#undef SHAFFT_ATTR
#define SHAFFT_PATTR(L, A, B, C_, NT)                                                            \
  if (e == cudaSuccess)                                                                          \
    e = cudaFuncSetAttribute(k_fft_plane<float, L, A, B, C_, NT>,                                \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
  SHAFFT_PLANE_LIST_F32(SHAFFT_PATTR)
#undef SHAFFT_PATTR
  return e;
}
#endif
#ifdef SHAFFT_INSTANTIATE_F64
template <>
cudaError_t fast_attr_all<double>() {
  cudaError_t e = cudaSuccess;
#define SHAFFT_ATTR(L, A, B, C_, NT)                                                             \
  if (e == cudaSuccess)                                                                          \
    e = cudaFuncSetAttribute(k_fft_fast<double, L, A, B, C_, NT, false>,                         \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);              \
  if (e == cudaSuccess)                                                                          \
    e = cudaFuncSetAttribute(k_fft_fast<double, L, A, B, C_, NT, true>,                          \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
  SHAFFT_FAST_LIST_F64(SHAFFT_ATTR)
#undef SHAFFT_ATTR
#define SHAFFT_PATTR(L, A, B, C_, NT)                                                            \
  if (e == cudaSuccess)                                                                          \
    e = cudaFuncSetAttribute(k_fft_plane<double, L, A, B, C_, NT>,                               \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
  SHAFFT_PLANE_LIST_F64(SHAFFT_PATTR)
#undef SHAFFT_PATTR
  return e;
}

#endif

template <typename T>
cudaError_t Launch<T>::init() {
  cudaError_t e = cudaFuncSetAttribute(k_fft_pass<T, 0, 0>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  return fast_attr_all<T>();
}



#ifdef SHAFFT_INSTANTIATE_F32
template <>
bool Launch<float>::fast_supported(int L) {
  switch (L) {
#define SHAFFT_CASE(L_, A, B, C_, NT) case L_: return true;
    SHAFFT_FAST_LIST_F32(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return false;
  }
}
template <>
int Launch<float>::fast_threads(int L) {
  switch (L) {
#define SHAFFT_CASE(L_, A, B, C_, NT) case L_: return NT;
    SHAFFT_FAST_LIST_F32(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return 0;
  }
}
template <>
cudaError_t Launch<float>::fast(const PassGeom& g, bool in_row, const C* in, C* out,
                                const PassTables<C>& tb, cudaStream_t s) {
  const unsigned grid = (unsigned)g.ntiles;
  switch (g.L) {
#define SHAFFT_CASE(L_, A, B, C_, NT)                                                          \
  case L_:                                                                                     \
    if (in_row)                                                                                \
      k_fft_fast<float, L_, A, B, C_, NT, true><<<grid, NT, L_ * 128, s>>>(g, in, out, tb);    \
    else                                                                                       \
      k_fft_fast<float, L_, A, B, C_, NT, false><<<grid, NT, L_ * 128, s>>>(g, in, out, tb);   \
    return cudaGetLastError();
    SHAFFT_FAST_LIST_F32(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return cudaErrorNotSupported;
  }
}
#endif
#ifdef SHAFFT_INSTANTIATE_F64
template <>
bool Launch<double>::fast_supported(int L) {
  switch (L) {
#define SHAFFT_CASE(L_, A, B, C_, NT) case L_: return true;
    SHAFFT_FAST_LIST_F64(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return false;
  }
}
template <>
int Launch<double>::fast_threads(int L) {
  switch (L) {
#define SHAFFT_CASE(L_, A, B, C_, NT) case L_: return NT;
    SHAFFT_FAST_LIST_F64(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return 0;
  }
}
template <>
cudaError_t Launch<double>::fast(const PassGeom& g, bool in_row, const C* in, C* out,
                                 const PassTables<C>& tb, cudaStream_t s) {
  const unsigned grid = (unsigned)g.ntiles;
  switch (g.L) {
#define SHAFFT_CASE(L_, A, B, C_, NT)                                                          \
  case L_:                                                                                     \
    if (in_row)                                                                                \
      k_fft_fast<double, L_, A, B, C_, NT, true><<<grid, NT, L_ * 128, s>>>(g, in, out, tb);   \
    else                                                                                       \
      k_fft_fast<double, L_, A, B, C_, NT, false><<<grid, NT, L_ * 128, s>>>(g, in, out, tb);  \
    return cudaGetLastError();
    SHAFFT_FAST_LIST_F64(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return cudaErrorNotSupported;
  }
}
#endif

#ifdef SHAFFT_INSTANTIATE_F32
template <>
bool Launch<float>::plane_supported(int L) {
  switch (L) {
#define SHAFFT_CASE(L_, A, B, C_, NT) case L_: return true;
    SHAFFT_PLANE_LIST_F32(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return false;
  }
}
template <>
cudaError_t Launch<float>::plane(const PassGeom& gx, const PassGeom& gy, const C* src, C* mid, C* dst,
                               const PassTables<C>& tb, int planes, int cluster, cudaStream_t s) {
  switch (gx.L) {
#define SHAFFT_CASE(L_, A, B, C_, NT)                                                            \
  case L_:                                                                                       \
    return launch_cluster(k_fft_plane<float, L_, A, B, C_, NT>, planes, cluster, NT, L_ * 128, s,  \
                          gx, gy, src, mid, dst, tb);
    SHAFFT_PLANE_LIST_F32(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return cudaErrorNotSupported;
  }
}
#endif

#ifdef SHAFFT_INSTANTIATE_F64
template <>
bool Launch<double>::plane_supported(int L) {
  switch (L) {
#define SHAFFT_CASE(L_, A, B, C_, NT) case L_: return true;
    SHAFFT_PLANE_LIST_F64(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return false;
  }
}
template <>
cudaError_t Launch<double>::plane(const PassGeom& gx, const PassGeom& gy, const C* src, C* mid, C* dst,
                               const PassTables<C>& tb, int planes, int cluster, cudaStream_t s) {
  switch (gx.L) {
#define SHAFFT_CASE(L_, A, B, C_, NT)                                                            \
  case L_:                                                                                       \
    return launch_cluster(k_fft_plane<double, L_, A, B, C_, NT>, planes, cluster, NT, L_ * 128, s,  \
                          gx, gy, src, mid, dst, tb);
    SHAFFT_PLANE_LIST_F64(SHAFFT_CASE)
#undef SHAFFT_CASE
    default: return cudaErrorNotSupported;
  }
}
#endif

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
