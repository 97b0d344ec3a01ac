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
//   row phase     warp w transforms rows w and w + 16 of its CTA's slab along
//                 the contiguous axis c (512 = 16 x 32): each lane loads the 16
//                 points c = lane + 32 m (coalesced 256-byte rows), DFT16 in
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
// cluster per plane at a time, as many clusters as fit on the GPU).  The only
// waits are the hardware cluster barriers, which every CTA of a cluster
// reaches the same number of times (all loop over the same planes), so no
// wait can hang.  No CTA touches another's shared memory after the last
// barrier it shares with it.  No bulk or tensor copies are used, so no load
// can multicast.  in == out is allowed: a plane's loads all complete before
// the first cluster barrier of that plane and its stores all come after it.
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
constexpr size_t kSmem = (size_t)kRows * kPL * sizeof(float2);  // 128 KiB
static_assert(kNT / 32 == 16 && kRows == 32, "the thread mapping assumes 16 warps and 32 rows");

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

__global__ void __launch_bounds__(kNT, 1)
    k_fft_plane_cluster(const float2* in, float2* out, int64_t planes, int64_t pstride_in,
                        int64_t pstride_out, const float2* __restrict__ tw, int conj_in, int conj_out,
                        float scale) {
  extern __shared__ __align__(128) float2 slab[];  // [kRows][kPL]
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int64_t ncl = gridDim.x / kCS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int col = rank * kRows + lane;  // this thread's column in the column phase

  for (int64_t P = blockIdx.x / kCS; P < planes; P += ncl) {
    __syncthreads();  // the previous plane's column phase is done with the slab
    // ---------------- row phase ----------------
    const float2* src = in + P * pstride_in + (int64_t)rank * kRows * kPL;
#pragma unroll 1
    for (int rr = 0; rr < 2; ++rr) {
      float2* row = slab + (warp + 16 * rr) * kPL;
      float2 v[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) v[m] = __ldcs(src + (warp + 16 * rr) * kPL + lane + 32 * m);
#pragma unroll
      for (int m = 0; m < 16; ++m)
        if (conj_in) v[m].y = -v[m].y;
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
    cl.sync();  // every slab holds its rows' transforms
    // ---------------- column phase ----------------
    float2 y[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) {
      const float2* rem = cl.map_shared_rank(slab, m >> 1);
      y[m] = rem[(warp + 16 * (m & 1)) * kPL + col];
    }
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
                               double scale, cudaStream_t s) {
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
                            conj_in, conj_out, (float)scale);
}

}  // namespace shafft_sm100
