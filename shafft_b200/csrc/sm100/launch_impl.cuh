// Definitions of Launch<T> (see launch.h); included by launch_f32.cu and
// launch_f64.cu only (each defines SHAFFT_INSTANTIATE_F32 or _F64).
#pragma once
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>

#include <cudaTypedefs.h>

#include "fast.cuh"
#include "fast_tma.cuh"
#include "kernels.cuh"
#include "launch.h"

namespace shafft_sm100 {

// 2-D grid of 256-thread blocks over `rows` rows of `len` points (block
// tiles of kEwUnroll*256 points): at most one wave of 8 blocks per SM, rows
// in y (<= 65535).
static inline dim3 row_grid(int64_t rows, int64_t len) {
  const int64_t cap = 148 * 8;
  const int64_t per = 256 * kEwUnroll;
  const int64_t gx = std::max<int64_t>(1, std::min<int64_t>((len + per - 1) / per, cap));
  const int64_t gy = std::max<int64_t>(1, std::min<int64_t>({rows, std::max<int64_t>(1, cap / gx), 65535}));
  return dim3((unsigned)gx, (unsigned)gy, 1);
}

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

// Column-tile passes fed by bulk tensor copies (k_fft_fast_tma):
// (L, R0, R1, R2, threads, stages, CTAs per SM).  Shared memory per CTA is
// stages x L x 128 bytes (3 x 64 KiB for L = 512: one CTA of 16 warps per SM;
// 3 x 32 KiB for L = 256: two CTAs of 8 warps).
#define SHAFFT_TMA_LIST(X)        \
  X(256, 8, 8, 4, 256, 3, 2)      \
  X(512, 8, 8, 8, 512, 3, 1)

// SHAFFT_SM100_TMA=1 turns the bulk-copy column passes on (default: the
// register-load k_fft_fast, which measured faster on B200: 512^3 complex64
// column pass 0.464 vs 0.534 ms, 2^24 complex64 FFT1D 0.418 vs 0.592 ms
// fwd+bwd; one CTA per SM cannot overlap its own barriers and butterflies
// the way three independent CTAs do).  SHAFFT_SM100_TMA_L2 = 0..3 picks the
// L2 promotion of the copies (none, 64, 128, 256 bytes; default 2; no
// measurable difference).
static bool tma_enabled() {
  static const bool on = [] {
    const char* e = getenv("SHAFFT_SM100_TMA");
    return e && atoi(e) != 0;
  }();
  return on;
}

static int tma_l2_promotion() {
  static const int v = [] {
    const char* e = getenv("SHAFFT_SM100_TMA_L2");
    const int x = e ? atoi(e) : 2;
    return (x >= 0 && x <= 3) ? x : 2;
  }();
  return v;
}

static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// Tensor map of a column pass's input (see fast_tma.cuh).  False when the
// view does not qualify (alignment, strides, extents); the caller then runs
// the register-load kernel.
static bool tma_map_for(const PassGeom& g, const void* in, int csize, CUtensorMap* map, TmaDims* d) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(in) & 15) || g.sin[0] != 1) return false;
  const int box_n = g.L < 256 ? g.L : 256;
  if (g.L % box_n) return false;
  // (index, extent, byte stride) of n, b1, b2, b3
  struct Ax {
    int id;
    int64_t ext, stride;
  } ax[4] = {{0, g.L, g.sn_in * csize}, {1, g.ext[1], g.sin[1] * csize}, {2, g.ext[2], g.sin[2] * csize},
             {3, g.ext[3], g.sin[3] * csize}};
  int64_t top = 16;
  for (const Ax& a : ax) {
    if (a.ext < 1 || a.ext > (int64_t)1 << 31) return false;
    if (a.ext > 1) {
      if (a.stride <= 0 || a.stride % 16) return false;
      top = std::max(top, a.stride * a.ext);
    }
  }
  // unit axes get a stride past every used one, so that strides ascend
  for (Ax& a : ax)
    if (a.ext == 1) a.stride = top;
  if (top >= (int64_t)1 << 40) return false;
  std::stable_sort(ax, ax + 4, [](const Ax& x, const Ax& y) { return x.stride < y.stride; });
  cuuint64_t dims[5], strides[4];
  cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
  dims[0] = (cuuint64_t)g.ext[0] * (csize / 4);
  box[0] = 32;
  if (dims[0] % 32 || dims[0] > ((cuuint64_t)1 << 32)) return false;
  int pos[4];
  for (int i = 0; i < 4; ++i) {
    dims[i + 1] = (cuuint64_t)ax[i].ext;
    strides[i] = (cuuint64_t)ax[i].stride;
    box[i + 1] = ax[i].id == 0 ? (cuuint32_t)box_n : 1u;
    pos[ax[i].id] = i + 1;
  }
  d->n = pos[0];
  d->b1 = pos[1];
  d->b2 = pos[2];
  d->b3 = pos[3];
  const CUtensorMapL2promotion l2[4] = {CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_64B,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<void*>(in), dims, strides, box,
                         estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         l2[tma_l2_promotion()], CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// SMs of the current device (queried per call: a process may drive devices
// of different sizes).
static unsigned sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    sms = 148;
  return (unsigned)std::max(1, sms);
}

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

// The extended instantiations of the specialised pass, k_fft_fast<..., EXT>:
// EXT_BS with the fused Bluestein loads and stores (complex64 plans only;
// PassGeom::bs_mode) and EXT_MAP with an exchange block map (map_mode).
// Plain passes launch the instantiation without either.
template <typename T, int L, int A, int B, int C_, int NT, int X>
static cudaError_t fast_ext_attr() {
  cudaError_t e = cudaFuncSetAttribute(k_fft_fast<T, L, A, B, C_, NT, true, X>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fft_fast<T, L, A, B, C_, NT, false, X>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
  return e;
}
template <typename T, int L, int A, int B, int C_, int NT, int X>
static cudaError_t fast_ext_launch(bool in_row, unsigned grid, const PassGeom& g, const typename Vec2<T>::type* in,
                                   typename Vec2<T>::type* out, const PassTables<typename Vec2<T>::type>& tb,
                                   cudaStream_t s) {
  if (in_row)
    k_fft_fast<T, L, A, B, C_, NT, true, X><<<grid, NT, L * 128, s>>>(g, in, out, tb);
  else
    k_fft_fast<T, L, A, B, C_, NT, false, X><<<grid, NT, L * 128, s>>>(g, in, out, tb);
  return cudaGetLastError();
}
template <typename T, int L, int A, int B, int C_, int NT>
struct FastExt {
  static cudaError_t attr() { return fast_ext_attr<T, L, A, B, C_, NT, EXT_MAP>(); }
  static cudaError_t launch(bool in_row, unsigned grid, const PassGeom& g, const typename Vec2<T>::type* in,
                            typename Vec2<T>::type* out, const PassTables<typename Vec2<T>::type>& tb,
                            cudaStream_t s) {
    if (g.bs_mode) return cudaErrorNotSupported;
    return fast_ext_launch<T, L, A, B, C_, NT, EXT_MAP>(in_row, grid, g, in, out, tb, s);
  }
};
template <int L, int A, int B, int C_, int NT>
struct FastExt<float, L, A, B, C_, NT> {
  static cudaError_t attr() {
    const cudaError_t e = fast_ext_attr<float, L, A, B, C_, NT, EXT_BS>();
    return e == cudaSuccess ? fast_ext_attr<float, L, A, B, C_, NT, EXT_MAP>() : e;
  }
  static cudaError_t launch(bool in_row, unsigned grid, const PassGeom& g, const float2* in, float2* out,
                            const PassTables<float2>& tb, cudaStream_t s) {
    if (g.bs_mode) return fast_ext_launch<float, L, A, B, C_, NT, EXT_BS>(in_row, grid, g, in, out, tb, s);
    return fast_ext_launch<float, L, A, B, C_, NT, EXT_MAP>(in_row, grid, g, in, out, tb, s);
  }
};

// L2 prefetch distance of k_fft_fast_pf, in quarter waves of resident CTAs
// (0 runs k_fft_fast).  Row-input (transposing) passes:
// SHAFFT_SM100_PREFETCH_ROW, default 4 (one wave); column-input passes:
// SHAFFT_SM100_PREFETCH_COL, default 0.  Only the complex64 512-point pass
// has a prefetching instantiation.  Measured on B200 (512^3 complex64
// fwd+bwd): one wave ahead on the row passes takes them from 0.433 to
// 0.39-0.40 ms each with per-launch timing and 2.56-2.62 -> 2.55-2.61 ms per
// step under graph replay; half a wave, 1.5 waves and 2 waves were slower
// than none (2.65-3.01 ms), prefetching the column pass slowed it (0.467 ->
// 0.502 ms), and the same kernel at L = 256 (256^3 complex128 and
// complex64, 2^24 complex64) lost 3-8%.
static int prefetch_quarters(bool in_row) {
  static const int v[2] = {[] {
                             const char* e = getenv("SHAFFT_SM100_PREFETCH_COL");
                             const int x = e ? atoi(e) : 0;
                             return (x >= 0 && x <= 32) ? x : 0;
                           }(),
                           [] {
                             const char* e = getenv("SHAFFT_SM100_PREFETCH_ROW");
                             const int x = e ? atoi(e) : 4;
                             return (x >= 0 && x <= 32) ? x : 4;
                           }()};
  return v[in_row ? 1 : 0];
}

// SHAFFT_SM100_BULK_PREFETCH (default 1): the row-input prefetches of
// k_fft_fast_pf as one bulk asynchronous prefetch per row (4 KiB for the
// complex64 512-point pass); 0: one prefetch per 128-byte line.  Measured on
// B200 (512^3 complex64, same box, two repetitions): 2.504 / 2.507 ms per
// step against 2.508 / 2.521 ms with the per-line prefetches.
static int bulk_prefetch() {
  static const int on = [] {
    const char* e = getenv("SHAFFT_SM100_BULK_PREFETCH");
    return (e && atoi(e) == 0) ? 0 : 1;
  }();
  return on;
}

// SHAFFT_SM100_COL_FETCH = 256 (default 0): the complex64 512-point passes
// with column input load with 256-byte L2 fetches (k_fft_fast_pf<..., 256>).
static bool col_fetch_256() {
  static const bool on = [] {
    const char* e = getenv("SHAFFT_SM100_COL_FETCH");
    return e && atoi(e) == 256;
  }();
  return on;
}

template <typename T, int L, int A, int B, int C_, int NT>
struct FastPf {
  static constexpr bool kOn = sizeof(T) == 4 && L == 512;
  static cudaError_t attr() {
    if constexpr (kOn) {
      cudaError_t e = cudaFuncSetAttribute(k_fft_fast_pf<T, L, A, B, C_, NT, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_fast_pf<T, L, A, B, C_, NT, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_fft_fast_pf<T, L, A, B, C_, NT, false, 256>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);
      return e;
    }
    return cudaSuccess;
  }
  // false: not taken (switched off, or no prefetching instantiation for L)
  static bool launch(bool in_row, unsigned grid, const PassGeom& g, const typename Vec2<T>::type* in,
                     typename Vec2<T>::type* out, const PassTables<typename Vec2<T>::type>& tb, cudaStream_t s) {
    if constexpr (kOn) {
      const int q = prefetch_quarters(in_row);
      const bool fetch = !in_row && col_fetch_256();
      if (q == 0 && !fetch) return false;
      // resident CTAs on the current device: its SMs x the CTAs per SM the
      // kernel is compiled for (its 64 KiB tile fits that many)
      const int64_t resident = (int64_t)sm_count() * fast_pf_min_blocks<T, L>();
      const int64_t ahead = q == 0 ? 0 : std::max<int64_t>(1, resident * q / 4);
      if (in_row)
        k_fft_fast_pf<T, L, A, B, C_, NT, true>
            <<<grid, NT, L * 128, s>>>(g, in, out, tb, ahead, bulk_prefetch());
      else if (fetch)
        k_fft_fast_pf<T, L, A, B, C_, NT, false, 256><<<grid, NT, L * 128, s>>>(g, in, out, tb, ahead, 0);
      else
        k_fft_fast_pf<T, L, A, B, C_, NT, false><<<grid, NT, L * 128, s>>>(g, in, out, tb, ahead, 0);
      return true;
    }
    return false;
  }
};

#define SHAFFT_DEFINE_PRECISION(TYPE, FASTLIST, PLANELIST)                                       \
  template <>                                                                                    \
  cudaError_t fast_attr_all<TYPE>() {                                                            \
    cudaError_t e = cudaSuccess;                                                                 \
    FASTLIST(SHAFFT_ATTR_FAST)                                                                   \
    PLANELIST(SHAFFT_ATTR_PLANE)                                                                 \
    SHAFFT_TMA_LIST(SHAFFT_ATTR_TMA)                                                             \
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
  int Launch<TYPE>::fast_prefetch(int L, bool in_row) {                                          \
    switch (L) {                                                                                 \
      FASTLIST(SHAFFT_CASE_PF)                                                                   \
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
                                 const PassTables<C>& tb, int* err, cudaStream_t s) {            \
    const unsigned grid = (unsigned)g.ntiles;                                                    \
    if (!in_row && err && !g.bs_mode && !g.map_mode && tma_enabled()) {                          \
      CUtensorMap map;                                                                           \
      TmaDims d;                                                                                 \
      switch (g.L) {                                                                             \
        SHAFFT_TMA_LIST(SHAFFT_CASE_TMA)                                                         \
        default: break;                                                                          \
      }                                                                                          \
    }                                                                                            \
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
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128);               \
  if (e == cudaSuccess) e = FastExt<TYPE_, L, A, B, C_, NT>::attr();                             \
  if (e == cudaSuccess) e = FastPf<TYPE_, L, A, B, C_, NT>::attr();
#define SHAFFT_ATTR_PLANE(L, A, B, C_, NT)                                                        \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_plane_flow<TYPE_, L, A, B, C_, NT>,                            \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L * 128 + 128);         \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_plane_flow<TYPE_, L, A, B, C_, NT>,                            \
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
#define SHAFFT_TMA_SMEM(L_, ST) ((size_t)(ST) * (L_) * 128 + 8 * (ST))
#define SHAFFT_ATTR_TMA(L_, A, B, C_, NT, ST, MB)                                                 \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_fast_tma<TYPE_, L_, A, B, C_, NT, ST, MB>,                         \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, SHAFFT_TMA_SMEM(L_, ST)); \
  if (e == cudaSuccess)                                                                           \
    e = cudaFuncSetAttribute(k_fft_fast_tma<TYPE_, L_, A, B, C_, NT, ST, MB>,                         \
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
#define SHAFFT_CASE_TMA(L_, A, B, C_, NT, ST, MB)                                                 \
  case L_:                                                                                        \
    if (tma_map_for(g, in, (int)sizeof(C), &map, &d)) {                                           \
      const unsigned tg = (unsigned)std::min<int64_t>(g.ntiles, (int64_t)sm_count() * (MB));      \
      k_fft_fast_tma<TYPE_, L_, A, B, C_, NT, ST, MB><<<tg, NT, SHAFFT_TMA_SMEM(L_, ST), s>>>(          \
          map, g, d, out, tb, err);                                                               \
      count_tma_launch();                                                                         \
      return cudaGetLastError();                                                                  \
    }                                                                                             \
    break;
#define SHAFFT_CASE_TRUE(L_, A, B, C_, NT) \
  case L_:                                 \
    return true;
#define SHAFFT_CASE_PF(L_, A, B, C_, NT) \
  case L_:                               \
    return FastPf<TYPE_, L_, A, B, C_, NT>::kOn ? prefetch_quarters(in_row) : 0;
#define SHAFFT_CASE_NT(L_, A, B, C_, NT) \
  case L_:                               \
    return NT;
#define SHAFFT_CASE_FAST(L_, A, B, C_, NT)                                                       \
  case L_:                                                                                       \
    if (g.bs_mode || g.map_mode) return FastExt<TYPE_, L_, A, B, C_, NT>::launch(in_row, grid, g, in, out, tb, s); \
    if (FastPf<TYPE_, L_, A, B, C_, NT>::launch(in_row, grid, g, in, out, tb, s)) return cudaGetLastError(); \
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
cudaError_t Launch<T>::init_device() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static bool done[kMaxDevices] = {};
  static cudaError_t result[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (!done[dev]) {
    result[dev] = init();
    done[dev] = true;
  }
  return result[dev];
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
  const int64_t rows = M > 0 ? total / M : 0;
  if (rows == 0) return cudaSuccess;
  k_bs_modulate<T><<<row_grid(rows, M), 256, 0, s>>>(src, dst, L, M, I, rows, chirp, conj);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::bs_mulh(C* d, const C* H, int64_t M, int64_t total, cudaStream_t s) {
  const int64_t rows = M > 0 ? total / M : 0;
  if (rows == 0) return cudaSuccess;
  k_bs_mulh<T><<<row_grid(rows, M), 256, 0, s>>>(d, H, M, rows);
  return cudaGetLastError();
}

template <typename T>
cudaError_t Launch<T>::bs_demod(const C* src, C* dst, int64_t L, int64_t M, int64_t I, int64_t total,
                                const C* chirp, int conj, T scale, cudaStream_t s) {
  const int64_t rows = L > 0 ? total / L : 0;
  if (rows == 0) return cudaSuccess;
  k_bs_demod<T><<<row_grid(rows, L), 256, 0, s>>>(src, dst, L, M, I, rows, chirp, conj, scale);
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
