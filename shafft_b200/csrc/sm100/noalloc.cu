// Allocation-free 1-D Bluestein transform: shafft_sm100_bluestein_noalloc.
//
// Some callers cannot call cudaMalloc at the point where they need a
// transform: code running under a memory-pool or allocator lock, a host
// that captured its device memory budget up front, or a framework that
// forbids allocations inside its compute callbacks.  The regular plan API
// allocates its tables and Bluestein scratch at plan time; this entry point
// instead keeps everything it needs in one file-scope __device__ array and
// takes only the caller's input and output buffers.
//
// Limits and sharing rules:
//   * 1 <= n <= kNoAllocMaxN (2048) complex elements; larger n is rejected
//     with SHAFFT_SM100_EINVAL before any device work.
//   * The array (kNoAllocBytes, about 304 KiB) lives on every device that
//     loads the library, until the process exits.
//   * Every call on a device reuses the same array and leaves the last
//     call's contents in it.  Each call regenerates all of its tables and
//     writes every scratch element it later reads (the zero padding of the
//     convolution rows included), so nothing depends on previous contents.
//   * Calls whose work overlaps on the GPU (different streams, or any
//     concurrency on the same device) race on the array and corrupt each
//     other; serialise them, e.g. by issuing them on one stream.
//   * The first call on a device resolves the array's device address with
//     cudaGetSymbolAddress (a runtime call made once per device), and the
//     first call of each precision on a device sets the pass kernels'
//     shared-memory limit there (cudaFuncSetAttribute, once per device and
//     precision); make those first calls before capturing a stream.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "../../../include/shafft_sm100.h"
#include "launch.h"
#include "pass.h"

namespace shafft_sm100 {

constexpr int64_t kNoAllocMaxN = 2048;
constexpr int64_t kNoAllocMaxM = 4096;  // power of two >= 2*kNoAllocMaxN - 1
// complex128-sized slots: chirp[N], H[M], twL[M], S0[M], S1[M]; then two
// uint16 digit tables of M entries
constexpr size_t kNoAllocSlots = (size_t)kNoAllocMaxN + 4 * (size_t)kNoAllocMaxM;
constexpr size_t kNoAllocBytes = kNoAllocSlots * 16 + 2 * 2 * (size_t)kNoAllocMaxM;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

int fail(int code, const char* fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  return report_error(code, msg);
}

// digit-reversal tables of the radix plan of L (same mapping as the
// planner's host-side tables)
__global__ void k_gen_digits(uint16_t* p2k, uint16_t* k2p, int L) {
  const RadixPlan rp = radix_plan(L);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < L; p += gridDim.x * blockDim.x) {
    int rem = p, k = 0, pre = 1, span = L;
    for (int s = 0; s < rp.n; ++s) {
      const int m = span / rp.r[s];
      const int d = rem / m;
      rem -= d * m;
      k += d * pre;
      pre *= rp.r[s];
      span = m;
    }
    p2k[p] = (uint16_t)k;
    k2p[k] = (uint16_t)p;
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_dev_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (resolved once
// per device).
int scratch_ptr(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SHAFFT_SM100_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(SHAFFT_SM100_ENOTSUP, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_dev_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(SHAFFT_SM100_ECUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_dev_ptr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_dev_ptr[dev]);
  return 0;
}

// One M-point forward pass over a single contiguous row (generic kernel).
PassGeom row_geom(int M, double scale) {
  PassGeom g{};
  const RadixPlan rp = radix_plan(M);
  g.L = M;
  g.nst = rp.n;
  for (int s = 0; s < rp.n; ++s) g.rad[s] = rp.r[s];
  g.W = 1;
  g.logW = 0;
  g.pitch = 1;
  g.in_row = g.out_row = 1;
  for (int d = 0; d < 4; ++d) {
    g.ext[d] = 1;
    g.sin[d] = g.sout[d] = 0;
  }
  g.sin[0] = g.sout[0] = M;
  g.sn_in = g.sk_out = 1;
  g.tiles_w = 1;
  g.ntiles = 1;
  g.tw_mode = TW_NONE;
  g.scale = scale;
  return g;
}

template <typename T>
int run(const void* in, void* out, int64_t n, int direction, double scale, cudaStream_t s,
        unsigned char* base) {
  using K = Launch<T>;
  using C = typename Vec2<T>::type;
  int64_t M = 1;
  while (M < 2 * n - 1) M <<= 1;
  if (M < 2) M = 2;
  C* slot = reinterpret_cast<C*>(base);
  const size_t stride = 16 / sizeof(C);  // slots are complex128-sized
  C* chirp = slot;
  C* H = slot + stride * kNoAllocMaxN;
  C* twL = H + stride * kNoAllocMaxM;
  C* S0 = twL + stride * kNoAllocMaxM;
  C* S1 = S0 + stride * kNoAllocMaxM;
  uint16_t* p2k = reinterpret_cast<uint16_t*>(base + kNoAllocSlots * 16);
  uint16_t* k2p = p2k + kNoAllocMaxM;

  cudaError_t e = K::init_device();
  if (e == cudaSuccess) e = K::gen_twiddle(twL, M, 1, M, s);
  if (e == cudaSuccess) {
    k_gen_digits<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(p2k, k2p, (int)M);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = K::gen_chirp(chirp, n, s);
  if (e == cudaSuccess) e = K::gen_bs_kernel(S0, chirp, n, M, s);
  PassTables<C> tb{};
  tb.twL = twL;
  tb.p2k = p2k;
  tb.k2p = k2p;
  const size_t smem = (size_t)M * sizeof(C);
  // H = FFT_M(h) / M
  if (e == cudaSuccess) e = K::pass(row_geom((int)M, 1.0 / (double)M), S0, H, tb, smem, s);
  // modulate (writes all M entries: the zero padding included)
  if (e == cudaSuccess)
    e = K::bs_modulate(reinterpret_cast<const C*>(in), S0, n, M, 1, M, chirp, direction, s);
  if (e == cudaSuccess) e = K::pass(row_geom((int)M, 1.0), S0, S1, tb, smem, s);
  if (e == cudaSuccess) e = K::bs_mulh(S1, H, M, M, s);
  if (e == cudaSuccess) e = K::pass(row_geom((int)M, 1.0), S1, S0, tb, smem, s);
  if (e == cudaSuccess)
    e = K::bs_demod(S0, reinterpret_cast<C*>(out), n, M, 1, n, chirp, direction, (T)scale, s);
  if (e != cudaSuccess) return fail(SHAFFT_SM100_ECUDA, "launch: %s", cudaGetErrorString(e));
  return 0;
}

}  // namespace
}  // namespace shafft_sm100

using namespace shafft_sm100;

extern "C" int shafft_sm100_bluestein_noalloc(const void* in, void* out, int64_t n, int precision,
                                              int direction, double scale, void* stream) {
  if (!in || !out) return fail(SHAFFT_SM100_EINVAL, "null buffer");
  if (n < 1 || n > kNoAllocMaxN)
    return fail(SHAFFT_SM100_EINVAL,
                "n = %lld is outside 1..%lld supported by the allocation-free entry point",
                (long long)n, (long long)kNoAllocMaxN);
  if (precision != 0 && precision != 1) return fail(SHAFFT_SM100_EINVAL, "bad precision");
  if (direction != 0 && direction != 1) return fail(SHAFFT_SM100_EINVAL, "bad direction");
  const uintptr_t align = precision ? 16 : 8;  // whole complex elements
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & (align - 1))
    return fail(SHAFFT_SM100_EINVAL, "buffers must be aligned to the complex element size");
  unsigned char* base = nullptr;
  int rc = scratch_ptr(&base);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return precision ? run<double>(in, out, n, direction, scale, s, base)
                   : run<float>(in, out, n, direction, scale, s, base);
}
