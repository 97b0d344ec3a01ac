// Definitions of Launch<T> (see launch.h); included by launch_f32.cu and
// launch_f64.cu only (each defines SHAFFT_INSTANTIATE_F32 or _F64).
#pragma once
#include <stdio.h>
#include <stdlib.h>

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

// Lengths with a fused two-axis plane kernel (k_fft_plane_flow).
#define SHAFFT_PLANE_LIST_F32(X) \
  X(128, 8, 4, 4, 128)           \
  X(256, 8, 8, 4, 256)           \
  X(512, 8, 8, 8, 256)           \
  X(1024, 8, 8, 16, 512)
#define SHAFFT_PLANE_LIST_F64(X) \
  X(128, 8, 4, 4, 128)           \
  X(256, 8, 8, 4, 128)           \
  X(512, 8, 8, 8, 256)

// Resident CTAs of `kernel` on the current device.
template <typename KernelT>
static unsigned resident_ctas(KernelT kernel, int threads, size_t smem) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  return (unsigned)(sms * per);
}

template <typename T, typename KernelT>
static cudaError_t launch_flow(KernelT kernel, int threads, size_t smem, const PassGeom& gx,
                               const PassGeom& gy, const typename Vec2<T>::type* src,
                               typename Vec2<T>::type* mid, typename Vec2<T>::type* dst,
                               const PassTables<typename Vec2<T>::type>& tb, int planes, int* ctl,
                               int lag, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(int) * (size_t)(4 + planes), s);
  if (e != cudaSuccess) return e;
  FlowShape f;
  f.planes = planes;
  f.tx = gx.tiles_w;
  f.ty = gy.tiles_w;
  f.lag = std::max(1, std::min(lag, planes));
  // cache policies: X tiles keep the intermediate in L2, Y tiles read it at
  // L2 and discard it; SHAFFT_SM100_FLOW_POLICY="xld,xst,yld,yst,discard"
  // overrides them (values of TileLoad / TileStore, discard 0/1)
  f.xpol = TilePolicy{LD_STREAM, ST_KEEP, 0};
  f.ypol = TilePolicy{LD_L2, ST_STREAM, 1};
  if (const char* env = getenv("SHAFFT_SM100_FLOW_POLICY")) {
    int v[5] = {LD_STREAM, ST_KEEP, LD_L2, ST_STREAM, 1};
    sscanf(env, "%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4]);
    f.xpol = TilePolicy{v[0], v[1], 0};
    f.ypol = TilePolicy{v[2], v[3], v[4]};
  }
  const unsigned grid = resident_ctas(kernel, threads, smem);
  kernel<<<grid, threads, smem, s>>>(gx, gy, src, mid, dst, tb, ctl, f);
  return cudaGetLastError();
}

#define SHAFFT_DEFINE_PRECISION(TYPE, FASTLIST, PLANELIST)                                       \
  template <>                                                                                    \
  cudaError_t fast_attr_all<TYPE>() {                                                            \
    cudaError_t e = cudaSuccess;                                                                 \
    FASTLIST(SHAFFT_ATTR_FAST)                                                                   \
    PLANELIST(SHAFFT_ATTR_PLANE)                                                                 \
    return e;                                                                                    \
  }                                                                                              \
  template <>                                                                                    \
  bool Launch<TYPE>::fast_supported(int L) {                                                     \
    switch (L) {                                                                                 \
      FASTLIST(SHAFFT_CASE_TRUE)                                                                 \
      default: return false;                                                                     \
    }                                                                                            \
  }                                                                                              \
  template <>                                                                                    \
  int Launch<TYPE>::fast_threads(int L) {                                                        \
    switch (L) {                                                                                 \
      FASTLIST(SHAFFT_CASE_NT)                                                                   \
      default: return 0;                                                                         \
    }                                                                                            \
  }                                                                                              \
  template <>                                                                                    \
  bool Launch<TYPE>::plane_supported(int L) {                                                    \
    switch (L) {                                                                                 \
      PLANELIST(SHAFFT_CASE_TRUE)                                                                \
      default: return false;                                                                     \
    }                                                                                            \
  }                                                                                              \
  template <>                                                                                    \
  cudaError_t Launch<TYPE>::fast(const PassGeom& g, bool in_row, const C* in, C* out,            \
                                 const PassTables<C>& tb, cudaStream_t s) {                      \
    const unsigned grid = (unsigned)g.ntiles;                                                    \
    switch (g.L) {                                                                               \
      FASTLIST(SHAFFT_CASE_FAST)                                                                 \
      default: return cudaErrorNotSupported;                                                     \
    }                                                                                            \
  }                                                                                              \
  template <>                                                                                    \
  cudaError_t Launch<TYPE>::plane(const PassGeom& gx, const PassGeom& gy, const C* src, C* mid,  \
                                  C* dst, const PassTables<C>& tb, int planes, int* ctl,        \
                                  int lag, cudaStream_t s) {                                     \
    switch (gx.L) {                                                                              \
      PLANELIST(SHAFFT_CASE_PLANE)                                                               \
      default: return cudaErrorNotSupported;                                                     \
    }                                                                                            \
  }

template <typename T>
static cudaError_t fast_attr_all();

#define SHAFFT_ATTR_FAST(L, A, B, C_, NT)                                                         \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_fast<TYPE_, L, A, B, C_, NT, true>,                            \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);               \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_fast<TYPE_, L, A, B, C_, NT, false>,                           \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
#define SHAFFT_ATTR_PLANE(L, A, B, C_, NT)                                                        \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_plane_flow<TYPE_, L, A, B, C_, NT>,                            \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128 + 128);         \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_plane_flow<TYPE_, L, A, B, C_, NT>,                            \
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
#define SHAFFT_CASE_TRUE(L_, A, B, C_, NT) \
  case L_:                                 \
    return true;
#define SHAFFT_CASE_NT(L_, A, B, C_, NT) \
  case L_:                               \
    return NT;
#define SHAFFT_CASE_FAST(L_, A, B, C_, NT)                                                       \
  case L_:                                                                                       \
    if (in_row)                                                                                  \
      k_fft_fast<TYPE_, L_, A, B, C_, NT, true><<<grid, NT, L_ * 128, s>>>(g, in, out, tb);      \
    else                                                                                         \
      k_fft_fast<TYPE_, L_, A, B, C_, NT, false><<<grid, NT, L_ * 128, s>>>(g, in, out, tb);     \
    return cudaGetLastError();
#define SHAFFT_CASE_PLANE(L_, A, B, C_, NT)                                                      \
  case L_:                                                                                       \
    return launch_flow<TYPE_>(k_fft_plane_flow<TYPE_, L_, A, B, C_, NT>, NT, L_ * 128 + 128, gx, \
                              gy, src, mid, dst, tb, planes, ctl, lag, s);

#ifdef SHAFFT_INSTANTIATE_F32
#define TYPE_ float
SHAFFT_DEFINE_PRECISION(float, SHAFFT_FAST_LIST_F32, SHAFFT_PLANE_LIST_F32)
#undef TYPE_
#endif
#ifdef SHAFFT_INSTANTIATE_F64
#define TYPE_ double
SHAFFT_DEFINE_PRECISION(double, SHAFFT_FAST_LIST_F64, SHAFFT_PLANE_LIST_F64)
#undef TYPE_
#endif

// Compile-time instances of the generic pass (length, tile width): the radix
// sequence and every index division fold into constants.  The lengths are
// the factors of the 3^5*5^3*7^2 = 1,488,375 FFT1D plan (1215 * 1225) at the
// tile widths its complex64 (4) and complex128 (2) plans use; measured on
// B200 the complex64 transform drops from 0.108 to 0.099 ms fwd+bwd.
#define SHAFFT_GENERIC_LIST(X) \
  X(1215, 4)                   \
  X(1225, 4)                   \
  X(1215, 2)                   \
  X(1225, 2)

template <typename T>
cudaError_t Launch<T>::init() {
  cudaError_t e = cudaFuncSetAttribute(k_fft_pass<T, 0, 0>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
#define SHAFFT_ATTR_GENERIC(L_, W_)                                                          \
  if (e == cudaSuccess)                                                                      \
    e = cudaFuncSetAttribute(k_fft_pass<T, L_, W_>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                             200 * 1024);
  SHAFFT_GENERIC_LIST(SHAFFT_ATTR_GENERIC)
#undef SHAFFT_ATTR_GENERIC
  if (e != cudaSuccess) return e;
  return fast_attr_all<T>();
}

template <typename T>
cudaError_t Launch<T>::pass(const PassGeom& g, const C* in, C* out, const PassTables<C>& tb,
                            size_t smem, cudaStream_t s) {
  const int64_t grid = std::min<int64_t>(g.ntiles, 148 * 64);
#define SHAFFT_CASE_GENERIC(L_, W_)                                                    \
  if (g.L == L_ && g.W == W_) {                                                        \
    k_fft_pass<T, L_, W_><<<(unsigned)grid, kThreads, smem, s>>>(g, in, out, tb);      \
    return cudaGetLastError();                                                         \
  }
  SHAFFT_GENERIC_LIST(SHAFFT_CASE_GENERIC)
#undef SHAFFT_CASE_GENERIC
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
