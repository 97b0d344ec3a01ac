// Specialised column-tile pass fed by the tensor-memory accelerator.
//
// Same arithmetic as k_fft_fast with IN_ROW = false (fast.cuh), but the
// input tile (L rows of one 128-byte column chunk) reaches shared memory by
// bulk tensor copies (cp.async.bulk.tensor, no multicast) instead of by
// register loads.  One persistent CTA per SM cycles through STAGES tile
// buffers: while its warps transform tile i in place, the copies of tiles
// i+1 .. i+STAGES-1 are in flight, so the load of the next tiles overlaps
// the butterflies and the stores of this one (the register-load kernel
// alternates those phases inside each CTA).
//
// Each stage has an mbarrier armed with the tile's byte count; every thread
// waits on it (bounded: after kTmaSpinLimit polls the CTA sets *err = 1,
// waits -- again bounded -- for the copies it still has in flight, and
// returns).  A buffer is refilled only after the whole CTA has finished
// reading it (barrier, then a proxy fence by the issuing thread).
//
// The tensor map describes the input view (element (n, b0..b3) at
// n*sn_in + sum b_d*sin[d]) as a rank-5 tensor of 4-byte words: dimension 0
// is the contiguous b0 axis, dimensions 1..4 are n, b1, b2, b3 in ascending
// stride order.  The box is 32 words (128 bytes) x min(L, 256) points, so a
// tile is L/256 copies (one for L <= 256) landing as dense 128-byte rows.
#pragma once
#include <cuda.h>

#include "fast.cuh"

namespace shafft_sm100 {

constexpr long long kTmaSpinLimit = 1ll << 22;  // mbarrier polls before giving up

// tensor-map dimension (1..4) of the pass's n, b1, b2, b3 indices
struct TmaDims {
  int n, b1, b2, b3;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool tma_wait(uint32_t bar, uint32_t parity) {
  uint32_t done = 0;
  for (long long i = 0; i < kTmaSpinLimit && !done; ++i) {
    asm volatile(
        "{\n\t.reg .pred q;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
  }
  return done != 0;
}

// Arm `bar` with the tile's bytes and issue the copies of tile `t` into the
// buffer at shared address `dst` (one thread).
template <int L>
__device__ __forceinline__ void tma_issue_tile(const CUtensorMap* map, const PassGeom& g, const TmaDims& d,
                                               int64_t t, uint32_t dst, uint32_t bar) {
  constexpr int BOX = L < 256 ? L : 256;
  constexpr int NBOX = L / BOX;
  const int64_t tw = t % g.tiles_w;
  int64_t rest = t / g.tiles_w;
  const int64_t i1 = rest % g.ext[1];
  rest /= g.ext[1];
  const int64_t i2 = rest % g.ext[2];
  const int64_t i3 = rest / g.ext[2];
  int c[5];
  c[0] = (int)(tw * 32);  // 128-byte chunk = 32 words: x stays 16-byte aligned
  c[d.b1] = (int)i1;
  c[d.b2] = (int)i2;
  c[d.b3] = (int)i3;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(L * 128)
               : "memory");
#pragma unroll
  for (int k = 0; k < NBOX; ++k) {
    c[d.n] = k * BOX;
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst + k * BOX * 128),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]),
        "r"(bar)
        : "memory");
  }
}

template <typename T, int L, int R0, int R1, int R2, int NT, int STAGES, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_fft_fast_tma(const __grid_constant__ CUtensorMap map, const __grid_constant__ PassGeom g,
                   const TmaDims d, typename Cx<T>::type* out,
                   const __grid_constant__ PassTables<typename Cx<T>::type> tb, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  constexpr int TILE = L * 128;
  const int tid = threadIdx.x;
  const uint32_t base = smem_addr(smem_raw);
  const uint32_t bar0 = base + STAGES * TILE;
  const int64_t ntiles = g.ntiles;
  const int64_t G = gridDim.x;
  if (base & 127) {  // a bulk tensor copy needs a 128-byte aligned buffer
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (tid == 0) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
    for (int s = 0; s < STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8 * s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int s = 0; s < STAGES; ++s) {
      const int64_t t = blockIdx.x + s * G;
      if (t < ntiles) tma_issue_tile<L>(&map, g, d, t, base + s * TILE, bar0 + 8 * s);
    }
  int64_t it = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += G, ++it) {
    const int s = (int)(it % STAGES);
    const bool ok = tma_wait(bar0 + 8 * s, (uint32_t)((it / STAGES) & 1));
    if (__syncthreads_or(!ok)) {
      // give up: report, then let the copies still in flight land before the
      // CTA (and its shared memory) goes away
      if (tid == 0) {
        atomicExch(err, 1);
        for (int64_t j = it; j < it + STAGES; ++j)
          if (blockIdx.x + j * G < ntiles) tma_wait(bar0 + 8 * (int)(j % STAGES), (uint32_t)((j / STAGES) & 1));
      }
      __syncthreads();
      return;
    }
    fast_tile<T, L, R0, R1, R2, NT, false, LD_STREAM, ST_STREAM, false, true>(
        g, nullptr, out, tb, t, reinterpret_cast<float4*>(smem_raw + s * TILE));
    __syncthreads();  // every read of this buffer is done
    if (tid == 0) {
      const int64_t nt = t + STAGES * G;
      if (nt < ntiles) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tma_issue_tile<L>(&map, g, d, nt, base + s * TILE, bar0 + 8 * s);
      }
    }
  }
}

}  // namespace shafft_sm100
