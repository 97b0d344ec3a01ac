// Tensor-core form of a complex64 FFT pass: one DFT stage of length L <= 64
// per pass, computed as dense GEMMs on the 5th-generation tensor cores.
//
// A pass runs batched length-L DFTs over an arbitrary set of rows (the
// PassGeom batch dims b0..b3 flattened).  A tile holds NG groups of 128 rows
// (NG = 4 for L <= 16, 2 for L <= 32, else 1), so that every tile moves about
// 64 KiB whatever L is; group j accumulates in TMEM columns [j*2Lp, (j+1)*2Lp):
//
//   y[m][k] = sum_n x[m][n] * w_L^{n k}          m < 128 rows, n, k < L
//
// in real arithmetic  yr = xr*Cr - xi*Ci,  yi = xr*Ci + xi*Cr  with
// C = w_L^{nk}.  Split precision recovers complex64 accuracy from FP16
// operands: every row of the tile is scaled by a power of two so that its
// largest component lands in [2^13, 2^14), then each value v is split into
// hi = fp16(v) and lo = fp16(v - hi) (22-23 significant bits together); the
// DFT matrix is split the same way.  The product keeps the three significant
// terms  hi*Chi + lo*Chi + hi*Clo  (the lo*lo term is below FP32 rounding),
// accumulated in FP32 in tensor memory.  Each tcgen05.mma is M=128 (rows),
// N = Lp (L padded to a multiple of 16), K = 16; 3 products x Lp/16 K-steps
// x 4 real GEMMs per group, issued by one thread, completion signalled by
// tcgen05.commit on an mbarrier.  The epilogue reads the accumulators with
// tcgen05.ld (warp w reads TMEM lanes 32*(w%4)..+31, i.e. one row per
// thread), undoes the row scale and fuses the four-step twiddle, the
// normalisation scale and the output conjugation into the store.
//
// Software pipeline: right after the MMAs of tile i are issued, every thread
// decodes the rows of tile i+1 and issues its global loads, so HBM reads of
// the next tile overlap the tensor-core work and the epilogue of this one.
//
// Shared memory operands use the no-swizzle K-major canonical layout: 8x8
// FP16 core matrices of 128 contiguous bytes (8 rows of 16 bytes); row
// groups 128 B apart (SBO), K-chunks of 8 elements R*16 B apart (LBO).
//
// FP64 is used only where the plan builds its tables (w_L, w_N).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <mutex>
#include <stdint.h>

#include "kernels.cuh"
#include "launch.h"
#include "pass.h"

namespace shafft_sm100 {
namespace {

constexpr int kTcRows = 128;
constexpr int kTcThreads = 256;
constexpr int kTcMaxLen = 64;
constexpr uint32_t kTcTmemCols = 128;
constexpr long long kTcSpinLimit = 1ll << 26;  // mbarrier polls before giving up

struct TcLayout {
  int Lp, NG, RT;  // padded length, 128-row groups per tile, rows per tile
  uint32_t a_bytes, b_bytes;
  uint32_t off_a, off_b, off_rows, off_max, off_bar, total;
};

// Row tables and row maxima are double-buffered: the next tile's rows are
// decoded and its inputs loaded while the current tile is on the tensor core.
__host__ __device__ inline TcLayout tc_layout(int L) {
  TcLayout t;
  t.Lp = (L + 15) & ~15;
  t.NG = t.Lp <= 16 ? 4 : (t.Lp <= 32 ? 2 : 1);
  t.RT = kTcRows * t.NG;
  t.a_bytes = (uint32_t)kTcRows * t.Lp * 2;   // one 128 x Lp FP16 operand
  t.b_bytes = (uint32_t)t.Lp * t.Lp * 2;      // one Lp x Lp FP16 operand
  t.off_a = 0;                                // per group: xr_hi, xr_lo, xi_hi, xi_lo
  t.off_b = 4 * t.NG * t.a_bytes;             // Cr_hi, Cr_lo, Ci_hi, Ci_lo
  t.off_rows = t.off_b + 4 * t.b_bytes;       // 2 x (row in, row out, twiddle index)
  t.off_max = t.off_rows + 2 * 3 * t.RT * 8;  // 2 x row maxima (float bits)
  t.off_bar = t.off_max + 2 * t.RT * 4;       // mbarrier, TMEM base, wait status
  t.total = t.off_bar + 16;
  return t;
}

// byte offset of the 16-byte chunk (row r, K-chunk c) of an R-row operand
__device__ __forceinline__ uint32_t cm_off(int r, int c, int R) {
  return (uint32_t)c * R * 16 + (uint32_t)(r >> 3) * 128 + (uint32_t)(r & 7) * 16;
}

// shared-memory matrix descriptor, no swizzle, K-major
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: FP16 A/B, FP32 D, both K-major, M = 128
__device__ __forceinline__ uint32_t instr_desc(int N, bool neg_b) {
  return (1u << 4) | ((neg_b ? 1u : 0u) << 14) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
  __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// v = hi + lo with hi = fp16(v), lo = fp16(v - hi)
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  __half2 h = __floats2half2_rn(a, b);
  const float2 hf = __half22float2(h);
  hi = *reinterpret_cast<uint32_t*>(&h);
  lo = pack_h2(a - hf.x, b - hf.y);
}

// 2^e as a float (e clamped to the normal range)
__device__ __forceinline__ float pow2f(int e) {
  e = e < -126 ? -126 : (e > 127 ? 127 : e);
  return __int_as_float((127 + e) << 23);
}

// exponent shift that brings a row maximum into [2^13, 2^14)
__device__ __forceinline__ int row_shift(uint32_t maxbits) {
  const float mx = __uint_as_float(maxbits);
  if (!(mx > 0.f)) return 0;
  int e;
  frexpf(mx, &e);  // mx = f * 2^e, f in [0.5, 1)
  return 14 - e;
}

struct TcRows {
  int64_t* in;
  int64_t* out;
  int64_t* t;
  uint32_t* max;
};

__device__ __forceinline__ TcRows tc_rows(unsigned char* smem, const TcLayout& ly, int b) {
  TcRows r;
  r.in = reinterpret_cast<int64_t*>(smem + ly.off_rows) + b * 3 * ly.RT;
  r.out = r.in + ly.RT;
  r.t = r.out + ly.RT;
  r.max = reinterpret_cast<uint32_t*>(smem + ly.off_max) + b * ly.RT;
  return r;
}

// rows of `tile`: input / output offsets and twiddle index
__device__ __forceinline__ void tc_decode(const PassGeom& g, const TcLayout& ly, int64_t tile,
                                          int64_t rows_total, const TcRows& R) {
  for (int i = threadIdx.x; i < ly.RT; i += kTcThreads) {
    int64_t r = tile * ly.RT + i;
    if (r < rows_total) {
      const int64_t b0 = r % g.ext[0];
      r /= g.ext[0];
      const int64_t b1 = r % g.ext[1];
      r /= g.ext[1];
      const int64_t b2 = r % g.ext[2];
      const int64_t b3 = r / g.ext[2];
      R.in[i] = b0 * g.sin[0] + b1 * g.sin[1] + b2 * g.sin[2] + b3 * g.sin[3];
      R.out[i] = b0 * g.sout[0] + b1 * g.sout[1] + b2 * g.sout[2] + b3 * g.sout[3];
      R.t[i] = g.tw_dim == 0 ? b0 : (g.tw_dim == 1 ? b1 : (g.tw_dim == 2 ? b2 : b3));
    } else {
      R.in[i] = -1;
      R.out[i] = -1;
      R.t[i] = 0;
    }
    R.max[i] = 0u;
  }
}

// item `it` = 8 consecutive n of one row (tile row r, K-chunk c).  Lanes
// walk rows in both orientations: the 16-byte operand stores of a warp then
// fill whole core matrices (no bank conflicts); for row tiles each lane reads
// 64 contiguous bytes of its row.
__device__ __forceinline__ void tc_item(const TcLayout& ly, int it, int& r, int& c) {
  r = it % ly.RT;
  c = it / ly.RT;
}

// issue every global load of the thread's items (no use before all issued)
__device__ __forceinline__ void tc_load(const PassGeom& g, const TcLayout& ly, const float2* in,
                                        const TcRows& R, int NI, float2 (&v)[4][8]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i >= NI) break;
    int m, c;
    tc_item(ly, threadIdx.x + i * kTcThreads, m, c);
    const int64_t base = R.in[m];
    const int n0 = 8 * c;
    if (g.in_row && base >= 0 && n0 + 8 <= g.L && ((base + n0) & 1) == 0) {
      // row tile, 16-byte aligned: four 16-byte loads of 2 elements
      const float4* src = reinterpret_cast<const float4*>(in + base + n0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float4 q = __ldcs(src + j);
        v[i][2 * j] = make_float2(q.x, q.y);
        v[i][2 * j + 1] = make_float2(q.z, q.w);
      }
      continue;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = n0 + j;
      float2 x = {0.f, 0.f};
      if (base >= 0 && n < g.L) x = __ldcs(in + base + (int64_t)n * g.sn_in);
      v[i][j] = x;
    }
  }
}

__global__ void __launch_bounds__(kTcThreads, 2)
    k_fft_tc(const __grid_constant__ PassGeom g, const float2* in, float2* out,
             const __grid_constant__ PassTables<float2> tb, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const TcLayout ly = tc_layout(g.L);
  const int L = g.L, Lp = ly.Lp, G = Lp / 8;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + ly.off_bar + 8);
  volatile uint32_t* wait_status = reinterpret_cast<uint32_t*>(smem + ly.off_bar + 12);
  const uint32_t s_base = (uint32_t)__cvta_generic_to_shared(smem);
  const uint32_t bar_addr = s_base + ly.off_bar;

  // tensor memory: 128 columns, one warp allocates
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     s_base + ly.off_bar + 8),
                 "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_addr));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // DFT matrix, split, built once per plan (k_gen_tc_dft): 16-byte copies
  {
    const uint4* src = static_cast<const uint4*>(tb.tcB);
    uint4* dst = reinterpret_cast<uint4*>(smem + ly.off_b);
    for (int i = tid; i < (int)(4 * ly.b_bytes / 16); i += kTcThreads) dst[i] = __ldg(src + i);
  }

  const int64_t rows_total = g.ext[0] * g.ext[1] * g.ext[2] * g.ext[3];
  const int64_t ntiles = (rows_total + ly.RT - 1) / ly.RT;
  const int NG = ly.NG;
  const int NI = (ly.RT * G) / kTcThreads;  // load items (8 elements of one row) per thread
  const float oscale = (float)g.scale;
  uint32_t phase = 0;
  int buf = 0;
  int64_t tile = blockIdx.x;
  float2 v[4][8];

  // prologue: rows and inputs of the first tile
  tc_decode(g, ly, tile, rows_total, tc_rows(smem, ly, 0));
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  if (tile < ntiles) tc_load(g, ly, in, tc_rows(smem, ly, 0), NI, v);

  while (tile < ntiles) {
    const TcRows R = tc_rows(smem, ly, buf);
    // input conjugation / pre-twiddle, row maxima
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (i >= NI) break;
      int r, c;
      tc_item(ly, tid + i * kTcThreads, r, c);
      float mx = 0.f;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float2 x = v[i][j];
        if (g.conj_in) x.y = -x.y;
        if (g.tw_mode == TW_PRE && R.in[r] >= 0 && 8 * c + j < L)
          x = cmul(x, tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)(8 * c + j) * R.t[r]));
        v[i][j] = x;
        mx = fmaxf(mx, fmaxf(fabsf(x.x), fabsf(x.y)));
      }
      atomicMax(&R.max[r], __float_as_uint(mx));
    }
    __syncthreads();
    // split into the four A operands of the row's group
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (i >= NI) break;
      int r, c;
      tc_item(ly, tid + i * kTcThreads, r, c);
      const float f = pow2f(row_shift(R.max[r]));
      uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        split2(v[i][j].x * f, v[i][j + 1].x * f, rh[j / 2], rl[j / 2]);
        split2(v[i][j].y * f, v[i][j + 1].y * f, ih[j / 2], il[j / 2]);
      }
      const uint32_t o = cm_off(r % kTcRows, c, kTcRows);
      unsigned char* A = smem + ly.off_a + (uint32_t)(r / kTcRows) * 4 * ly.a_bytes;
      *reinterpret_cast<uint4*>(A + 0 * ly.a_bytes + o) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
      *reinterpret_cast<uint4*>(A + 1 * ly.a_bytes + o) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
      *reinterpret_cast<uint4*>(A + 2 * ly.a_bytes + o) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
      *reinterpret_cast<uint4*>(A + 3 * ly.a_bytes + o) = make_uint4(il[0], il[1], il[2], il[3]);
    }
    // make the generic-proxy shared stores visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();

    if (tid == 0) {
      fence_after_sync();
      const uint32_t idp = instr_desc(Lp, false), idn = instr_desc(Lp, true);
      const uint32_t lbo_a = (uint32_t)kTcRows * 16, lbo_b = (uint32_t)Lp * 16;
      const uint64_t dA = smem_desc(s_base + ly.off_a, lbo_a, 128);
      const uint64_t dB = smem_desc(s_base + ly.off_b, lbo_b, 128);
      // start addresses stay below 2^18, so offsets add into the 14-bit field
      for (int gi = 0; gi < NG; ++gi) {
        const uint32_t t_re = tmem + (uint32_t)(gi * 2 * Lp), t_im = t_re + (uint32_t)Lp;
        const uint32_t ga = (uint32_t)gi * 4 * ly.a_bytes;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          const uint32_t ai = (p == 1) ? 1u : 0u;  // A lo for the second product
          const uint32_t bi = (p == 2) ? 1u : 0u;  // C lo for the third
          for (int s = 0; s < Lp / 16; ++s) {
            const uint32_t acc = (p | s) ? 1u : 0u;
            const uint64_t aR = dA + ((ga + (0 + ai) * ly.a_bytes + 2 * s * lbo_a) >> 4);
            const uint64_t aI = dA + ((ga + (2 + ai) * ly.a_bytes + 2 * s * lbo_a) >> 4);
            const uint64_t bR = dB + (((0 + bi) * ly.b_bytes + 2 * s * lbo_b) >> 4);
            const uint64_t bI = dB + (((2 + bi) * ly.b_bytes + 2 * s * lbo_b) >> 4);
            mma_f16(t_re, aR, bR, idp, acc);
            mma_f16(t_re, aI, bI, idn, 1u);
            mma_f16(t_im, aR, bI, idp, acc);
            mma_f16(t_im, aI, bR, idp, 1u);
          }
        }
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              bar_addr)
          : "memory");
    }

    // while the tensor core works: rows and inputs of the next tile
    const int64_t next = tile + gridDim.x;
    const TcRows RN = tc_rows(smem, ly, buf ^ 1);
    tc_decode(g, ly, next, rows_total, RN);
    __syncthreads();
    if (next < ntiles) tc_load(g, ly, in, RN, NI, v);

    // wait for the accumulators (one thread polls, bounded)
    if (tid == 0) {
      uint32_t done = 0;
      long long spins = 0;
      while (!done && spins++ < kTcSpinLimit) {
        asm volatile(
            "{\n\t.reg .pred q;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, q;\n\t}\n"
            : "=r"(done)
            : "r"(bar_addr), "r"(phase)
            : "memory");
      }
      *wait_status = done;
      if (!done) atomicExch(err, 1);
    }
    __syncthreads();
    if (!*wait_status) break;  // uniform: every thread read the same word
    phase ^= 1u;
    fence_after_sync();

    // epilogue: warp w reads TMEM lanes 32*(w%4)..; the two warp halves
    // (w/4) split the groups (NG >= 2) or the columns of the group (NG == 1)
    {
      const int q = warp & 3, h = warp >> 2;
      const int m = 32 * q + lane;
      const uint32_t lane_addr = tmem + ((uint32_t)(32 * q) << 16);
      const int g_lo = NG >= 2 ? h * (NG / 2) : 0, g_hi = NG >= 2 ? (h + 1) * (NG / 2) : 1;
      const int c_lo = NG >= 2 ? 0 : h * (G / 2), c_hi = NG >= 2 ? G : (h + 1) * (G / 2);
      for (int gi = g_lo; gi < g_hi; ++gi) {
        const int r = gi * kTcRows + m;
        const int64_t ob = R.out[r];
        const float f = pow2f(-row_shift(R.max[r])) * oscale;
        const int64_t t = R.t[r];
        // four-step twiddle w_N^{k t} = w_N^{k0 t} * w_N^{j t}, k = k0 + j:
        // the eight w_N^{j t} once per row, one table product per 8 outputs
        const bool post = g.tw_mode == TW_POST && ob >= 0;
        float2 wj[8];
        if (post) {
#pragma unroll
          for (int j = 0; j < 8; ++j) wj[j] = tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)j * t);
        }
        const uint32_t col = (uint32_t)(gi * 2 * Lp);
        for (int ck = c_lo; ck < c_hi; ++ck) {
          const int k0 = 8 * ck;
          float2 wb = {1.f, 0.f};
          if (post) wb = tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)k0 * t);
          float yr[8], yi[8];
          tmem_ld8(lane_addr + col + (uint32_t)k0, yr);
          tmem_ld8(lane_addr + col + (uint32_t)(Lp + k0), yi);
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
          if (ob >= 0) {
            float2 y[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              y[j] = make_float2(yr[j] * f, yi[j] * f);
              if (post) y[j] = cmul(y[j], cmul(wb, wj[j]));
              if (g.conj_out) y[j].y = -y[j].y;
            }
            if (g.out_row && k0 + 8 <= L && ((ob + k0) & 1) == 0) {
              // row tile, 16-byte aligned: four 16-byte stores
              float4* dst = reinterpret_cast<float4*>(out + ob + k0);
#pragma unroll
              for (int j = 0; j < 4; ++j)
                __stcs(dst + j, make_float4(y[2 * j].x, y[2 * j].y, y[2 * j + 1].x, y[2 * j + 1].y));
            } else {
#pragma unroll
              for (int j = 0; j < 8; ++j)
                if (k0 + j < L) __stcs(out + ob + (int64_t)(k0 + j) * g.sk_out, y[j]);
            }
          }
        }
      }
    }
    fence_before_sync();
    __syncthreads();  // TMEM and the A operands are reused by the next tile
    tile = next;
    buf ^= 1;
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTcTmemCols));
  }
}

// The split DFT matrix of length L in the shared-memory layout of k_fft_tc
// (four Lp x Lp FP16 operands Cr_hi, Cr_lo, Ci_hi, Ci_lo, K-major core
// matrices): element (k, n) = w_L^{nk} with the phase nk mod L reduced in
// integers and sincospi in FP64, zero outside L x L.
__global__ void k_gen_tc_dft(unsigned char* dst, int L) {
  const TcLayout ly = tc_layout(L);
  const int Lp = ly.Lp, G = Lp / 8;
  for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < G * Lp; it += gridDim.x * blockDim.x) {
    const int k = it % Lp, c = it / Lp;
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      float w[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = 8 * c + j + h;
        if (k < L && n < L) {
          double s, co;
          sincospi(-2.0 * (double)((n * k) % L) / (double)L, &s, &co);
          w[h][0] = (float)co;
          w[h][1] = (float)s;
        }
      }
      split2(w[0][0], w[1][0], rh[j / 2], rl[j / 2]);
      split2(w[0][1], w[1][1], ih[j / 2], il[j / 2]);
    }
    const uint32_t o = cm_off(k, c, Lp);
    *reinterpret_cast<uint4*>(dst + 0 * ly.b_bytes + o) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<uint4*>(dst + 1 * ly.b_bytes + o) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    *reinterpret_cast<uint4*>(dst + 2 * ly.b_bytes + o) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
    *reinterpret_cast<uint4*>(dst + 3 * ly.b_bytes + o) = make_uint4(il[0], il[1], il[2], il[3]);
  }
}

uint32_t tc_max_smem() {
  uint32_t m = 0;
  for (int L = 16; L <= kTcMaxLen; L += 16) m = tc_layout(L).total > m ? tc_layout(L).total : m;
  return m;
}

}  // namespace

bool tc_supported(const PassGeom& g) { return g.L >= 2 && g.L <= kTcMaxLen; }

size_t tc_smem_bytes(int L) { return tc_layout(L).total; }

size_t tc_table_bytes(int L) { return 4 * (size_t)tc_layout(L).b_bytes; }

int tc_gen_table(void* dst, int L, cudaStream_t s) {
  if (L < 2 || L > kTcMaxLen) return report_error(4, "tensor-core table: length outside 2..64");
  k_gen_tc_dft<<<8, 256, 0, s>>>(static_cast<unsigned char*>(dst), L);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : report_error(3, cudaGetErrorString(e));
}

int tc_pass(const PassGeom& g, const float2* in, float2* out, const PassTables<float2>& tb, int* err,
            cudaStream_t s) {
  if (!tc_supported(g)) return report_error(4, "tensor-core pass: length outside 2..64");
  constexpr int kMaxDev = 64;
  static std::mutex mu;
  static int sms[kMaxDev] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev)
    return report_error(3, "tensor-core pass: device query failed");
  std::unique_lock<std::mutex> lk(mu);
  if (!sms[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaFuncSetAttribute(k_fft_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc_max_smem()) != cudaSuccess)
      return report_error(3, "tensor-core pass: kernel set-up failed");
    sms[dev] = n;
  }
  const int nsm = sms[dev];
  lk.unlock();
  const TcLayout ly = tc_layout(g.L);
  const int64_t rows = g.ext[0] * g.ext[1] * g.ext[2] * g.ext[3];
  const int64_t ntiles = (rows + ly.RT - 1) / ly.RT;
  const int64_t grid = ntiles < 2 * (int64_t)nsm ? ntiles : 2 * (int64_t)nsm;
  if (grid < 1) return 0;
  k_fft_tc<<<(unsigned)grid, kTcThreads, ly.total, s>>>(g, in, out, tb, err);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return report_error(3, cudaGetErrorString(e));
  return 0;
}

}  // namespace shafft_sm100
