// Two axes of a stack of 512 x 512 complex64 planes in ONE HBM pass: a
// 16-CTA thread-block cluster holds a whole plane (2 MiB) in its distributed
// shared memory.
//
// A plane cannot be transformed along both of its axes inside one SM (2 MiB
// of data against 227 KB of shared memory), so the reference's slab
// machinery -- and the plain plans of this library -- spend two HBM passes
// on it (rows, then columns through a transposing store).  Here the 16 CTAs
// of a cluster split the plane into slabs of 32 rows (128 KiB each) and
// exchange the intermediate through distributed shared memory (DSMEM)
// instead of HBM:
//
//   prefetch      the first 24 rows of the CTA's slab of its NEXT plane are
//                 brought into a second shared buffer (96 KiB) by bulk copies
//                 (cp.async.bulk, this GPU's memory, no multicast) on an
//                 mbarrier while the current plane is being transformed; the
//                 other 8 rows are loaded by the warps that need them;
//   row phase     warp w transforms rows w and w + 16 of its CTA's slab along
//                 the contiguous axis c (512 = 16 x 32): each lane takes the 16
//                 points c = lane + 32 m (256 contiguous bytes per warp), DFT16 in
//                 registers, twiddle w512^(lane k1), a swizzled write of the
//                 16 x 32 block into its own slab row, DFT16 over l = 2 l2 + h
//                 per lane pair, radix-2 between the two lanes of a pair
//                 (shuffle), and the row's 512 outputs in natural order back
//                 into the slab row;
//   cluster barrier;
//   column phase  thread (w, lane) of CTA r owns column c = 32 r + lane and
//                 the 32 points b = w + 16 m of it, read from the slabs of
//                 CTAs m / 2 through DSMEM (each warp load is 256 contiguous
//                 bytes of one remote row); DFT32 in registers, twiddle
//                 w512^(w k1); after a second cluster barrier (no CTA reads
//                 another's slab any more) the 16 x 32 x 32 block goes through
//                 the CTA's own shared memory so that each thread gathers the
//                 16 values of one k1 over w, DFT16, and stores the outputs
//                 kb = k1 + 32 k2 with scale / conjugation fused, 256
//                 contiguous bytes per warp store.
//
// Every plane is read and written exactly once; the kernel is persistent (one
// cluster per plane at a time, as many clusters as fit on the GPU).  The
// cluster barriers are reached the same number of times by every CTA of a
// cluster (all loop over the same planes).  The prefetch wait is bounded:
// after kPreSpinLimit polls the CTA records *err = 1, carries on (its
// results are then wrong, never out of bounds) and, before exiting, waits --
// bounded again -- for the copy it may still have in flight.  No CTA touches
// another's shared memory after the last barrier it shares with it.
// in == out is allowed: every load of a plane (prefetch included) completes
// before the first cluster barrier of that plane, and its stores all come
// after it.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <mutex>

#include "butterflies.cuh"
#include "launch.h"
#include "pass.h"

namespace cg = cooperative_groups;

namespace shafft_sm100 {
namespace {

constexpr int kPL = 512;            // plane side
constexpr int kCS = 16;             // CTAs per cluster (non-portable size)
constexpr int kRows = kPL / kCS;    // 32 rows of the plane per CTA
constexpr int kNT = 512;            // threads per CTA: 16 warps
constexpr int kPre = 24;            // rows of the next plane prefetched by bulk copies
constexpr int kPreCopies = 6;       // bulk copies per prefetch (16 KiB each)
constexpr size_t kSlabBytes = (size_t)kRows * kPL * sizeof(float2);  // 128 KiB
constexpr size_t kPreBytes = (size_t)kPre * kPL * sizeof(float2);    // 96 KiB
constexpr size_t kSmem = kSlabBytes + kPreBytes + 16;                // + mbarrier
constexpr long long kPreSpinLimit = 1ll << 22;  // mbarrier polls before giving up
static_assert(kNT / 32 == 16 && kRows == 32, "the thread mapping assumes 16 warps and 32 rows");
static_assert(kPre >= 16 && kPre <= kRows && (kPreBytes / kPreCopies) % 16 == 0, "prefetch shape");

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// 8-byte load from the shared memory of CTA `rank` of this cluster, at the
// offset that `local` (a shared::cta address of this CTA) has in its own
__device__ __forceinline__ float2 ld_dsmem(uint32_t local, int rank) {
  uint32_t remote;
  float2 v;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(remote) : "memory");
  return v;
}

// bounded wait for phase `parity` of the mbarrier at `bar`; false on timeout
__device__ __forceinline__ bool pre_wait(uint32_t bar, uint32_t parity) {
  uint32_t done = 0;
  for (long long i = 0; i < kPreSpinLimit && !done; ++i) {
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

// one thread: arm the mbarrier with the prefetch's bytes and copy the first
// kPre rows of this CTA's slab of a plane into the prefetch buffer
__device__ __forceinline__ void pre_issue(const float2* rows, uint32_t dst, uint32_t bar) {
  constexpr uint32_t chunk = (uint32_t)(kPreBytes / kPreCopies);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"((uint32_t)kPreBytes)
               : "memory");
#pragma unroll
  for (int i = 0; i < kPreCopies; ++i)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            dst + i * chunk),
        "l"(reinterpret_cast<const char*>(rows) + (size_t)i * chunk), "r"(chunk), "r"(bar)
        : "memory");
}

// Row phase of one row: x[m] = the row's points c = lane + 32 m.  Leaves the
// row's 512 outputs in natural order in `row` (warp-private).
__device__ __forceinline__ void row_fft(float2* v, float2* row, const float2* __restrict__ tw, int lane) {
  dft16(v);  // over m: index k1
#pragma unroll
  for (int k1 = 1; k1 < 16; ++k1) v[k1] = cmul(v[k1], __ldg(tw + lane * k1));
  // Z[l = lane][k1] at k1*32 + (l ^ 2k1): conflict-free here and in the
  // strided gather below
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) row[k1 * 32 + (lane ^ ((2 * k1) & 31))] = v[k1];
  __syncwarp();
  const int k1p = lane >> 1, h = lane & 1;
#pragma unroll
  for (int l2 = 0; l2 < 16; ++l2) v[l2] = row[k1p * 32 + ((2 * l2 + h) ^ ((2 * k1p) & 31))];
  dft16(v);  // over l2: index k2a
  if (h) {
#pragma unroll
    for (int k2a = 1; k2a < 16; ++k2a) v[k2a] = cmul(v[k2a], __ldg(tw + 16 * k2a));
  }
#pragma unroll
  for (int k2a = 0; k2a < 16; ++k2a) {
    float2 o;
    o.x = __shfl_xor_sync(0xffffffffu, v[k2a].x, 1);
    o.y = __shfl_xor_sync(0xffffffffu, v[k2a].y, 1);
    v[k2a] = h ? csub(o, v[k2a]) : cadd(v[k2a], o);
  }
  __syncwarp();
  // X[k1p + 16 k2a + 256 h] in natural order
#pragma unroll
  for (int k2a = 0; k2a < 16; ++k2a) row[k1p + 16 * k2a + 256 * h] = v[k2a];
}

__global__ void __launch_bounds__(kNT, 1)
    k_fft_plane_cluster(const float2* in, float2* out, int64_t planes, int64_t pstride_in,
                        int64_t pstride_out, const float2* __restrict__ tw, int conj_in, int conj_out,
                        float scale, int* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float2* slab = reinterpret_cast<float2*>(smem_raw);               // [kRows][kPL]
  float2* pre = reinterpret_cast<float2*>(smem_raw + kSlabBytes);   // [kPre][kPL]
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(smem_raw + kSlabBytes + kPreBytes);
  const uint32_t pre_s = (uint32_t)__cvta_generic_to_shared(pre);
  const uint32_t slab_s = (uint32_t)__cvta_generic_to_shared(slab);
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int64_t ncl = gridDim.x / kCS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int col = rank * kRows + lane;  // this thread's column in the column phase
  const int64_t P0 = blockIdx.x / kCS;
  bool failed = false;

  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (P0 < planes) pre_issue(in + P0 * pstride_in + (int64_t)rank * kRows * kPL, pre_s, bar);
  }
  __syncthreads();

  uint32_t parity = 0;
  for (int64_t P = P0; P < planes; P += ncl, parity ^= 1) {
    // ---------------- row phase ----------------
    // rows warp (prefetched) and warp + 16 (prefetched below kPre, else
    // loaded from HBM now, before the wait, to overlap its latency)
    const float2* src = in + P * pstride_in + (int64_t)rank * kRows * kPL;
    const int r1 = warp + 16;
    float2 x[16], v[16];
    if (r1 >= kPre) {
#pragma unroll
      for (int m = 0; m < 16; ++m) x[m] = __ldcs(src + r1 * kPL + lane + 32 * m);
    }
    if (!pre_wait(bar, parity)) failed = true;
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = pre[warp * kPL + lane + 32 * m];
    if (r1 < kPre) {
#pragma unroll
      for (int m = 0; m < 16; ++m) x[m] = pre[r1 * kPL + lane + 32 * m];
    }
    __syncthreads();  // the prefetch buffer is consumed; the slab is free
    if (threadIdx.x == 0 && P + ncl < planes) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      pre_issue(in + (P + ncl) * pstride_in + (int64_t)rank * kRows * kPL, pre_s, bar);
    }
    if (conj_in) {
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        v[m].y = -v[m].y;
        x[m].y = -x[m].y;
      }
    }
    row_fft(v, slab + warp * kPL, tw, lane);
    row_fft(x, slab + r1 * kPL, tw, lane);
    cl.sync();  // every slab holds its rows' transforms
    // ---------------- column phase ----------------
    float2 y[32];
#pragma unroll
    for (int m = 0; m < 32; ++m)
      y[m] = ld_dsmem(slab_s + (uint32_t)(((warp + 16 * (m & 1)) * kPL + col) * sizeof(float2)), m >> 1);
    dft32(y);  // over m: index k1
    cluster_arrive();  // this CTA has read every slab it needs
#pragma unroll
    for (int k1 = 1; k1 < 32; ++k1) y[k1] = cmul(y[k1], __ldg(tw + warp * k1));
    cluster_wait();  // nobody reads this CTA's slab any more
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) slab[(warp * 32 + k1) * 32 + lane] = y[k1];
    __syncthreads();
    float2* dst = out + P * pstride_out;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int k1 = 2 * warp + q;
      float2 z[16];
#pragma unroll
      for (int w = 0; w < 16; ++w) z[w] = slab[(w * 32 + k1) * 32 + lane];
      dft16(z);  // over w: index k2
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) {
        float2 t = z[k2];
        if (scale != 1.0f) t = cscale(t, scale);
        if (conj_out) t.y = -t.y;
        __stcs(dst + (int64_t)(k1 + 32 * k2) * kPL + col, t);
      }
    }
    __syncthreads();  // the slab is free for the next plane's rows
  }
  if (failed) {
    atomicExch(err, 1);
    // a copy may still be in flight after a wait that gave up: wait for it
    // (bounded again) before the CTA's shared memory goes away
    pre_wait(bar, parity ^ 1);
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int g_state[kMaxDevices];     // 0 unknown, 1 ready, -1 unavailable
int g_clusters[kMaxDevices];  // co-resident clusters

// Per device: raise the kernel's shared-memory limit, allow the 16-CTA
// cluster and ask how many such clusters fit at once.
int setup(int* clusters) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return -1;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_state[dev] == 0) {
    int n = 0;
    cudaError_t e = cudaFuncSetAttribute(k_fft_plane_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_fft_plane_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = kCS;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      cfg.blockDim = dim3(kNT);
      cfg.gridDim = dim3(kCS);
      cfg.dynamicSmemBytes = kSmem;
      e = cudaOccupancyMaxActiveClusters(&n, (const void*)k_fft_plane_cluster, &cfg);
    }
    if (e != cudaSuccess || n < 1) {
      cudaGetLastError();
      g_state[dev] = -1;
    } else {
      g_state[dev] = 1;
      g_clusters[dev] = n;
    }
  }
  *clusters = g_clusters[dev];
  return g_state[dev];
}

}  // namespace

bool plane_cluster_len(int precision, int64_t L) { return precision == 0 && L == kPL; }

bool plane_cluster_available() {
  int n = 0;
  return setup(&n) == 1;
}

size_t plane_cluster_smem() { return kSmem; }

cudaError_t plane_cluster_pass(const float2* in, float2* out, int64_t planes, int64_t pstride_in,
                               int64_t pstride_out, const float2* tw, int conj_in, int conj_out,
                               double scale, int* err, cudaStream_t s) {
  int clusters = 0;
  if (setup(&clusters) != 1) return cudaErrorNotSupported;
  if (planes < 1) return cudaSuccess;
  const int64_t ncl = planes < clusters ? planes : clusters;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = kCS;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3(kNT);
  cfg.gridDim = dim3((unsigned)(ncl * kCS));
  cfg.dynamicSmemBytes = kSmem;
  cfg.stream = s;
  return cudaLaunchKernelEx(&cfg, k_fft_plane_cluster, in, out, planes, pstride_in, pstride_out, tw,
                            conj_in, conj_out, (float)scale, err);
}

}  // namespace shafft_sm100
