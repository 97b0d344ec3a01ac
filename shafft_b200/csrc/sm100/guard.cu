// Guard bytes around device allocations: a debugging safety net for
// out-of-bounds writes (SHAFFT_SM100_CANARY=1).
//
// With the switch on, every buffer that shafft_sm100_malloc returns and every
// table / scratch block a plan allocates gets kGuard bytes of a fixed pattern
// in front of it and behind it (the caller's pointer keeps its 256-byte
// alignment).  shafft_sm100_free and plan destruction check both guards of
// the block they release, and shafft_sm100_check_guards checks every live
// block; a changed byte means a kernel wrote outside the buffer it was
// given.  Checking reads the guards back with synchronous copies, so call it
// with the device idle.  With the switch off (the default) allocations are
// plain cudaMalloc / cudaFree.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <vector>

#include "../../../include/shafft_sm100.h"
#include "launch.h"

namespace shafft_sm100 {
namespace {

constexpr size_t kGuard = 256;
constexpr unsigned char kPattern = 0xA5;

struct Block {
  unsigned char* base;
  size_t bytes;
};

std::mutex g_mu;
std::map<void*, Block>& blocks() {
  static std::map<void*, Block> m;
  return m;
}

// 0 if both guards of b hold the pattern; otherwise a message in msg
int check_block(void* user, const Block& b, char* msg, size_t len) {
  std::vector<unsigned char> h(2 * kGuard);
  if (cudaMemcpy(h.data(), b.base, kGuard, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(h.data() + kGuard, b.base + kGuard + b.bytes, kGuard, cudaMemcpyDeviceToHost) !=
          cudaSuccess) {
    cudaGetLastError();
    snprintf(msg, len, "guard read-back failed for the buffer at %p", user);
    return SHAFFT_SM100_ECUDA;
  }
  for (size_t i = 0; i < 2 * kGuard; ++i)
    if (h[i] != kPattern) {
      const bool front = i < kGuard;
      snprintf(msg, len, "out-of-bounds write: guard byte %zu %s the %zu-byte buffer at %p was changed",
               front ? kGuard - i : i - kGuard + 1, front ? "before" : "after", b.bytes, user);
      return SHAFFT_SM100_ECUDA;
    }
  return 0;
}

}  // namespace

bool guard_enabled() {
  static const bool on = [] {
    const char* e = getenv("SHAFFT_SM100_CANARY");
    return e && atoi(e) != 0;
  }();
  return on;
}

cudaError_t dev_malloc(void** ptr, size_t bytes) {
  if (!guard_enabled()) return cudaMalloc(ptr, bytes);
  unsigned char* base = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&base), bytes + 2 * kGuard);
  if (e != cudaSuccess) return e;
  e = cudaMemset(base, kPattern, kGuard);
  if (e == cudaSuccess) e = cudaMemset(base + kGuard + bytes, kPattern, kGuard);
  if (e != cudaSuccess) {
    cudaFree(base);
    return e;
  }
  *ptr = base + kGuard;
  std::lock_guard<std::mutex> lk(g_mu);
  blocks()[*ptr] = Block{base, bytes};
  return cudaSuccess;
}

int dev_free(void* ptr) {
  if (!ptr) return 0;
  if (!guard_enabled()) {
    const cudaError_t e = cudaFree(ptr);
    if (e != cudaSuccess) return report_error(SHAFFT_SM100_ECUDA, cudaGetErrorString(e));
    return 0;
  }
  Block b;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = blocks().find(ptr);
    if (it == blocks().end()) return report_error(SHAFFT_SM100_EINVAL, "free of an unknown device pointer");
    b = it->second;
    blocks().erase(it);
  }
  char msg[256];
  const int rc = check_block(ptr, b, msg, sizeof(msg));
  cudaFree(b.base);
  return rc ? report_error(rc, msg) : 0;
}

}  // namespace shafft_sm100

extern "C" int shafft_sm100_check_guards(void) {
  using namespace shafft_sm100;
  if (!guard_enabled()) return 0;
  std::vector<std::pair<void*, Block>> live;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    live.assign(blocks().begin(), blocks().end());
  }
  char msg[256];
  for (const auto& kv : live) {
    const int rc = check_block(kv.first, kv.second, msg, sizeof(msg));
    if (rc) return report_error(rc, msg);
  }
  return 0;
}
