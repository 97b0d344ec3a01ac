// Batched form: thousands of independent C2C transforms of different shapes
// in ONE persistent kernel launch, replayed from a captured CUDA graph.
//
// Each transform (any rank, every axis of length <= 4096 with prime factors
// <= 13, or <= 362 for the direct-DFT path) is a sequence of passes, one per
// axis, src -> dst then in place on dst.  Every (transform, pass) is a "slot"
// with a device descriptor (PassGeom + table pointers).  Work tickets are
// handed out from one global counter.  The transforms are grouped into
// windows of about 16 MiB, and the ticket order is software-pipelined over
// them: stage s holds pass p of window s - p for every p, so a window's pass
// p runs one stage after its pass p-1, while that data is still in L2.  A
// tile of pass p of transform t first waits until every tile of pass p-1 of
// t has completed (per-slot counters, bounded wait).  Because every ticket
// of pass p-1 of t precedes every ticket of pass p of t and tickets are only
// claimed by running CTAs, every wait ends; the bound only guards against a
// fault elsewhere (it sets the batch's error flag and moves on).
//
// Tile shapes come from a small autotuner: for each distinct (precision,
// length, orientation) it times the candidate tile widths on a synthetic
// tensor the first time it meets the key and caches the winner in a text
// file (SHAFFT_SM100_TUNE_CACHE, default ~/.cache/shafft_sm100_tune.txt).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../../include/shafft_sm100.h"
#include "kernels.cuh"
#include "launch.h"
#include "pass.h"

namespace shafft_sm100 {
namespace {

int bfail(int code, const char* fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  return report_error(code, msg);
}

#define BCUDA(expr)                                                                    \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess) return bfail(SHAFFT_SM100_ECUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
  } while (0)

constexpr unsigned kBatchSpinLimit = 1u << 22;
// transforms per ticket-order window, in bytes (SHAFFT_SM100_BATCH_WINDOW_MB)
constexpr int64_t kBatchWindowBytes = int64_t(16) << 20;
// largest batch (in tiles) given a ticket -> slot table (4 bytes a ticket)
constexpr int64_t kMaxTicketTable = int64_t(1) << 26;
constexpr int64_t kBatchDirectMax = 362;  // the plans' direct-DFT range (plan.cu)
// tile widths (batch columns a tile holds): the autotuner's range and the
// defaults of axes it has not timed
constexpr int kBatchRowWMax = 256, kBatchColWMax = 64;
constexpr int kBatchRowWDefault = 256, kBatchColWDefault = 64;

// 16-byte aligned so that a warp copies each slot's PassGeom as int4s
template <typename C>
struct alignas(16) SlotDesc {
  PassGeom g;
  const C* twL;
  const uint16_t* p2k;
  const uint16_t* k2p;
  int transform;
  int pass;
  int last;  // 1 for the transform's final pass
  int prev;  // slot of the same transform's previous pass, or -1
  int need;  // tiles of that previous pass (its completion count)
};

int pow2_floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}

bool smooth13(int64_t L) {
  const int64_t primes[] = {2, 3, 5, 7, 11, 13};
  for (int64_t p : primes)
    while (L % p == 0) L /= p;
  return L == 1;
}

// slot of ticket t: the ticket table when there is one, else the last slot
// whose start <= t (binary search)
__device__ __forceinline__ int ticket_slot(long long t, const int* tslot, const int64_t* start, int nslots) {
  if (tslot) return tslot[t];
  int lo = 0, hi = nslots - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// One CTA works through tickets until the counter passes the last one.
// Thread 0 claims a ticket and finds its slot (a table lookup), waits for the
// slot's previous pass, and warp 0 copies the slot's geometry to shared
// memory with all its lanes.
// complex64: at most 80 registers so that three CTAs share an SM (the tiles
// are latency-bound; 116 registers allowed only two); complex128 unbounded
template <typename T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 3 : 1)
    k_fft_batch(const SlotDesc<typename Cx<T>::type>* slots, const int64_t* start, const int* tslot, int nslots,
                typename Cx<T>::type* const* src, typename Cx<T>::type* const* dst, int* done,
                unsigned long long* ticket, int* err, int conj, double scale, unsigned spin_limit) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  __shared__ __align__(16) PassGeom sg;
  __shared__ long long s_t;
  __shared__ int s_slot;
  static_assert(sizeof(PassGeom) % 16 == 0 && sizeof(PassGeom) / 16 <= 32, "one int4 per lane");
  static_assert(sizeof(SlotDesc<C>) % 16 == 0 && offsetof(SlotDesc<C>, g) == 0, "aligned slot geometry");
  const int64_t total = start[nslots];
  for (;;) {
    if (threadIdx.x == 0) {
      const long long t = (long long)atomicAdd(ticket, 1ull);
      s_t = t;
      int slot = -1;
      if (t < total) {
        slot = ticket_slot(t, tslot, start, nslots);
        const int pv = slots[slot].prev;
        if (pv >= 0) {
          const int need = slots[slot].need;
          unsigned it = 0;
          for (;;) {
            int v;
            asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(done + pv) : "memory");
            if (v >= need) break;
            if (++it > spin_limit) {
              atomicExch(err, 1);
              break;
            }
            __nanosleep(64);
          }
        }
      }
      s_slot = slot;
    }
    __syncthreads();
    const int slot = s_slot;
    if (slot < 0) break;
    const SlotDesc<C>& d = slots[slot];
    if (threadIdx.x < 32) {
      if (threadIdx.x < sizeof(PassGeom) / 16)
        reinterpret_cast<int4*>(&sg)[threadIdx.x] = reinterpret_cast<const int4*>(&d.g)[threadIdx.x];
      __syncwarp();
      if (threadIdx.x == 0) {
        sg.conj_in = (conj && d.pass == 0) ? 1 : 0;
        sg.conj_out = (conj && d.last) ? 1 : 0;
        sg.scale = d.last ? scale : 1.0;
      }
    }
    __syncthreads();
    PassTables<C> tb{};
    tb.twL = d.twL;
    tb.p2k = d.p2k;
    tb.k2p = d.k2p;
    C* o = dst[d.transform];
    const C* in = (d.pass == 0) ? src[d.transform] : o;
    generic_tile<T, 0, 0>(sg, in, o, tb, s_t - start[slot], sm);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(done + slot, 1);
    }
  }
}

// ---------------------------------------------------------------------------
// autotuner cache
// ---------------------------------------------------------------------------
std::mutex g_tune_mu;
std::map<std::string, int> g_tune;
bool g_tune_loaded = false;

std::string tune_path() {
  if (const char* e = getenv("SHAFFT_SM100_TUNE_CACHE")) return e;
  const char* home = getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/shafft_sm100_tune.txt";
}

void tune_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  FILE* f = fopen(tune_path().c_str(), "r");
  if (!f) return;
  char key[128];
  int w;
  while (fscanf(f, "%127s %d", key, &w) == 2) g_tune[key] = w;
  fclose(f);
}

void tune_store(const std::string& key, int w) {
  g_tune[key] = w;
  const std::string path = tune_path();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    std::string dir = path.substr(0, slash);
    std::string cmd = "mkdir -p '" + dir + "' 2>/dev/null";
    if (system(cmd.c_str()) != 0) return;
  }
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return;
  for (auto& kv : g_tune) fprintf(f, "%s %d\n", kv.first.c_str(), kv.second);
  fclose(f);
}

}  // namespace
}  // namespace shafft_sm100

using namespace shafft_sm100;

struct shafft_sm100_batch_s {
  int precision = 0;
  int count = 0;
  std::vector<int> ndims;
  std::vector<int64_t> dims;      // flattened
  std::vector<int64_t> elements;  // per transform
  int nslots = 0;
  int64_t tickets = 0;
  int64_t alg_bytes = 0;
  size_t smem = 0;
  unsigned grid = 0;
  // device memory
  unsigned char* d_tables = nullptr;  // twiddle + digit tables per distinct length
  void* d_slots = nullptr;
  int64_t* d_start = nullptr;
  int* d_tslot = nullptr;  // slot of every ticket (null above kMaxTicketTable tickets)
  int* d_ctl = nullptr;  // [0..1] ticket, [2] error, [4..4+nslots) done counters
  void** d_src = nullptr;
  void** d_dst = nullptr;
  // host copies of the last pointer sets + cached graph
  std::vector<void*> h_src, h_dst;
  cudaGraphExec_t graph = nullptr;
  int graph_conj = -1;
  double graph_scale = 0;
  cudaStream_t graph_stream = nullptr;
  // polls of a tile's wait for the previous pass before it gives up, sets
  // the error word and goes on (shafft_sm100_batch_set_wait_limit)
  unsigned wait_limit = kBatchSpinLimit;
  std::string desc;
};

namespace {

struct LenTab {
  size_t off_tw, off_p2k, off_k2p;
};

template <typename T>
int tune_width(int64_t L, bool row, int64_t ext0, int default_w, size_t es, int autotune) {
  const int maxw_smem = (int)std::max<int64_t>(1, (96 * 1024) / ((L + 1) * (int64_t)es));
  std::vector<int> cands;
  // widest tiles: 256 for rows, 64 for columns (the synthetic column tensor
  // has 64 columns), and at most 8192 points a tile
  const int wmax = row ? kBatchRowWMax : kBatchColWMax;
  for (int w = 1; w <= wmax; w *= 2) {
    if (w > maxw_smem || (w > 1 && (int64_t)w * L > 8192)) break;
    if (!row && w < 4 && ext0 >= 4) continue;
    if (w > 1 && w / 2 >= ext0) break;
    cands.push_back(w);
  }
  if (cands.empty()) return default_w;
  const std::string key = std::string(es == 8 ? "c64" : "c128") + ":L=" + std::to_string(L) +
                          (row ? ":row" : ":col");
  std::lock_guard<std::mutex> lk(g_tune_mu);
  tune_load();
  auto it = g_tune.find(key);
  if (it != g_tune.end()) return it->second;
  if (!autotune) return default_w;
  // time each candidate on a synthetic tensor of about 8 MiB
  using C = typename Vec2<T>::type;
  const int64_t n = std::max<int64_t>(L * 64, (8 << 20) / (int64_t)es);
  const int64_t rows = n / L;
  C *a = nullptr, *b = nullptr, *tw = nullptr;
  uint16_t* dg = nullptr;
  if (cudaMalloc(&a, rows * L * es) != cudaSuccess || cudaMalloc(&b, rows * L * es) != cudaSuccess ||
      cudaMalloc(&tw, L * es) != cudaSuccess || cudaMalloc(&dg, 4 * L) != cudaSuccess) {
    cudaGetLastError();
    if (a) cudaFree(a);
    if (b) cudaFree(b);
    if (tw) cudaFree(tw);
    return default_w;
  }
  cudaMemset(a, 0, rows * L * es);
  Launch<T>::init();
  Launch<T>::gen_twiddle(tw, L, 1, L, nullptr);
  PassTables<C> tb{};
  tb.twL = tw;
  tb.p2k = dg;
  tb.k2p = dg + L;
  cudaMemset(dg, 0, 4 * L);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best = default_w;
  float best_ms = 1e30f;
  for (int w : cands) {
    PassGeom g{};
    RadixPlan rp = radix_plan((int)L);
    g.L = (int)L;
    g.nst = rp.n > 0 ? rp.n : 0;
    for (int s = 0; s < g.nst; ++s) g.rad[s] = rp.r[s];
    g.W = w;
    g.logW = 0;
    while ((1 << g.logW) < w) ++g.logW;
    g.pitch = generic_pitch(w, row);
    if (row) {
      g.ext[0] = rows;
      g.sin[0] = g.sout[0] = L;
      g.sn_in = g.sk_out = 1;
    } else {
      g.ext[0] = 64;  // 64 columns, rows / 64 outer blocks
      g.sin[0] = g.sout[0] = 1;
      g.ext[1] = rows / 64;
      g.sin[1] = g.sout[1] = L * 64;
      g.sn_in = g.sk_out = 64;
    }
    for (int d = 0; d < 4; ++d)
      if (g.ext[d] < 1) g.ext[d] = 1;
    g.tiles_w = (g.ext[0] + w - 1) / w;
    g.ntiles = g.tiles_w * g.ext[1] * g.ext[2] * g.ext[3];
    g.in_row = row ? 1 : 0;
    g.out_row = row ? 1 : 0;
    g.scale = 1.0;
    const size_t smem = (size_t)L * g.pitch * es;
    float ms = 0;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(e0);
      Launch<T>::pass(g, a, b, tb, smem, nullptr);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      if (rep > 0) ms += t;  // first run warms up
    }
    if (cudaGetLastError() != cudaSuccess) continue;
    if (ms < best_ms) {
      best_ms = ms;
      best = w;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  cudaFree(tw);
  cudaFree(dg);
  tune_store(key, best);
  return best;
}

void digit_tables_host(int L, std::vector<uint16_t>& p2k, std::vector<uint16_t>& k2p) {
  RadixPlan rp = radix_plan(L);
  p2k.assign(L, 0);
  k2p.assign(L, 0);
  if (rp.n <= 0) return;
  for (int p = 0; p < L; ++p) {
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

template <typename T>
int batch_build(shafft_sm100_batch_s* b, int autotune) {
  using C = typename Vec2<T>::type;
  const size_t es = sizeof(C);
  int64_t window_bytes = kBatchWindowBytes;
  if (const char* e = getenv("SHAFFT_SM100_BATCH_WINDOW_MB")) window_bytes = (int64_t)atoll(e) << 20;
  // distinct lengths -> table offsets
  std::map<int64_t, LenTab> lens;
  size_t table_bytes = 0;
  auto alloc = [&](size_t bytes) {
    size_t off = (table_bytes + 255) & ~size_t(255);
    table_bytes = off + bytes;
    return off;
  };
  struct HostSlot {
    PassGeom g;
    int64_t L;
    int transform, pass, last, prev;
  };
  std::vector<std::vector<HostSlot>> per_transform(b->count);
  size_t maxsmem = 0;
  const int64_t* dp = b->dims.data();
  for (int t = 0; t < b->count; ++t) {
    const int nd = b->ndims[t];
    const int64_t* dims = dp;
    dp += nd;
    int pass = 0;
    for (int a = nd - 1; a >= 0; --a) {
      const int64_t L = dims[a];
      if (L == 1) continue;
      if (!(smooth13(L) && L <= 4096) && !(L <= kBatchDirectMax))
        return bfail(SHAFFT_SM100_ENOTSUP, "batch transform %d: axis length %lld not supported", t,
                     (long long)L);
      int64_t I = 1, O = 1;
      for (int c = a + 1; c < nd; ++c) I *= dims[c];
      for (int c = 0; c < a; ++c) O *= dims[c];
      HostSlot hs{};
      PassGeom& g = hs.g;
      RadixPlan rp = radix_plan((int)L);
      g.L = (int)L;
      g.nst = rp.n > 0 ? rp.n : 0;
      for (int s = 0; s < g.nst; ++s) g.rad[s] = rp.r[s];
      const bool row = (I == 1);
      int W;
      if (row) {
        // tile widths are powers of two (the tile walks columns by mask and shift)
        const int def = pow2_floor((int)std::min<int64_t>(kBatchRowWDefault, std::max<int64_t>(1, 8192 / L)));
        W = tune_width<T>(L, true, O, def, es, autotune);
        g.ext[0] = O;
        g.sin[0] = g.sout[0] = L;
        g.ext[1] = g.ext[2] = g.ext[3] = 1;
        g.sn_in = g.sk_out = 1;
      } else {
        const int def = pow2_floor((int)std::min<int64_t>(kBatchColWDefault, std::max<int64_t>(1, 8192 / L)));
        W = tune_width<T>(L, false, I, def, es, autotune);
        g.ext[0] = I;
        g.sin[0] = g.sout[0] = 1;
        g.ext[1] = O;
        g.sin[1] = g.sout[1] = L * I;
        g.ext[2] = g.ext[3] = 1;
        g.sn_in = g.sk_out = I;
      }
      // never wider than the batch dimension rounded up to a power of two
      int cap = 1;
      while (cap < g.ext[0] && cap < kBatchRowWMax) cap *= 2;
      W = std::max(1, std::min(W, cap));
      g.W = W;
      g.logW = 0;
      while ((1 << g.logW) < W) ++g.logW;
      g.pitch = generic_pitch(W, row);
      g.tiles_w = (g.ext[0] + W - 1) / W;
      g.ntiles = g.tiles_w * g.ext[1] * g.ext[2] * g.ext[3];
      g.in_row = row ? 1 : 0;
      g.out_row = row ? 1 : 0;
      g.scale = 1.0;
      maxsmem = std::max(maxsmem, (size_t)L * g.pitch * es);
      if (!lens.count(L)) lens[L] = LenTab{alloc(es * L), alloc(2 * L), alloc(2 * L)};
      hs.L = L;
      hs.transform = t;
      hs.pass = pass++;
      per_transform[t].push_back(hs);
    }
    if (per_transform[t].empty()) {
      // all axes of length 1: a single "pass" of length 1 copies the data
      HostSlot hs{};
      PassGeom& g = hs.g;
      g.L = 1;
      g.nst = 0;
      g.W = 1;
      g.pitch = 1;
      int64_t n = 1;
      for (int c = 0; c < nd; ++c) n *= dims[c];
      g.ext[0] = n;
      g.sin[0] = g.sout[0] = 1;
      g.ext[1] = g.ext[2] = g.ext[3] = 1;
      g.sn_in = g.sk_out = 1;
      g.tiles_w = n;
      g.ntiles = n;
      g.in_row = g.out_row = 1;
      g.scale = 1.0;
      if (!lens.count(1)) lens[1] = LenTab{alloc(es), alloc(2), alloc(2)};
      hs.L = 1;
      hs.transform = t;
      hs.pass = 0;
      per_transform[t].push_back(hs);
    }
    per_transform[t].back().last = 1;
  }
  // Ticket order.  The transforms are cut, in submission order, into
  // windows of about window_bytes; stage s holds pass p of window s - p for
  // every p, later passes first.  A window's next pass then follows its
  // previous one by one stage, while that data is still in L2, and every
  // slot still follows its previous pass in ticket order (the waits end).
  // One window (window_bytes = 0) is the pass-major order.
  std::vector<HostSlot> order;
  std::vector<std::vector<int>> slot_of(b->count);
  int maxpass = 0;
  for (auto& v : per_transform) maxpass = std::max(maxpass, (int)v.size());
  std::vector<int> wbeg{0};
  {
    int64_t acc = 0;
    for (int t = 0; t < b->count; ++t) {
      acc += b->elements[t] * (int64_t)es;
      if (window_bytes > 0 && acc >= window_bytes && t + 1 < b->count) {
        wbeg.push_back(t + 1);
        acc = 0;
      }
    }
    wbeg.push_back(b->count);
  }
  const int nwin = (int)wbeg.size() - 1;
  for (int st = 0; st < nwin + maxpass - 1; ++st)
    for (int p = maxpass - 1; p >= 0; --p) {
      const int w = st - p;
      if (w < 0 || w >= nwin) continue;
      for (int t = wbeg[w]; t < wbeg[w + 1]; ++t)
        if (p < (int)per_transform[t].size()) {
          HostSlot hs = per_transform[t][p];
          hs.prev = (p == 0) ? -1 : slot_of[t][p - 1];
          slot_of[t].push_back((int)order.size());
          order.push_back(hs);
        }
    }
  b->nslots = (int)order.size();
  std::vector<int64_t> start(order.size() + 1, 0);
  for (size_t i = 0; i < order.size(); ++i) start[i + 1] = start[i] + order[i].g.ntiles;
  b->tickets = start.back();
  b->alg_bytes = 0;
  for (auto& hs : order) {
    int64_t n = hs.g.L;
    for (int d = 0; d < 4; ++d) n *= hs.g.ext[d];
    b->alg_bytes += 2 * n * (int64_t)es;
  }
  // device allocations
  BCUDA(cudaMalloc(&b->d_tables, std::max<size_t>(table_bytes, 256)));
  BCUDA(cudaMalloc(&b->d_slots, sizeof(SlotDesc<C>) * order.size()));
  BCUDA(cudaMalloc(&b->d_start, sizeof(int64_t) * start.size()));
  BCUDA(cudaMalloc(&b->d_ctl, sizeof(int) * (4 + order.size())));
  BCUDA(cudaMalloc(&b->d_src, sizeof(void*) * b->count));
  BCUDA(cudaMalloc(&b->d_dst, sizeof(void*) * b->count));
  // tables
  BCUDA(Launch<T>::init());
  for (auto& kv : lens) {
    const int L = (int)kv.first;
    BCUDA(Launch<T>::gen_twiddle(reinterpret_cast<C*>(b->d_tables + kv.second.off_tw), L, 1,
                                 std::max(L, 1), nullptr));
    std::vector<uint16_t> p2k, k2p;
    digit_tables_host(L, p2k, k2p);
    BCUDA(cudaMemcpy(b->d_tables + kv.second.off_p2k, p2k.data(), 2 * L, cudaMemcpyHostToDevice));
    BCUDA(cudaMemcpy(b->d_tables + kv.second.off_k2p, k2p.data(), 2 * L, cudaMemcpyHostToDevice));
  }
  std::vector<SlotDesc<C>> hd(order.size());
  for (size_t i = 0; i < order.size(); ++i) {
    const HostSlot& hs = order[i];
    const LenTab& lt = lens[hs.L];
    hd[i].g = hs.g;
    hd[i].twL = reinterpret_cast<const C*>(b->d_tables + lt.off_tw);
    hd[i].p2k = reinterpret_cast<const uint16_t*>(b->d_tables + lt.off_p2k);
    hd[i].k2p = reinterpret_cast<const uint16_t*>(b->d_tables + lt.off_k2p);
    hd[i].transform = hs.transform;
    hd[i].pass = hs.pass;
    hd[i].last = hs.last;
    hd[i].prev = hs.prev;
    hd[i].need = hs.prev >= 0 ? (int)order[hs.prev].g.ntiles : 0;
  }
  BCUDA(cudaMemcpy(b->d_slots, hd.data(), sizeof(SlotDesc<C>) * hd.size(), cudaMemcpyHostToDevice));
  BCUDA(cudaMemcpy(b->d_start, start.data(), sizeof(int64_t) * start.size(), cudaMemcpyHostToDevice));
  // SHAFFT_SM100_BATCH_TICKET_TABLE=0 leaves the table out (the binary
  // search that batches above kMaxTicketTable tickets use)
  const char* tt = getenv("SHAFFT_SM100_BATCH_TICKET_TABLE");
  if (b->tickets <= kMaxTicketTable && !(tt && atoi(tt) == 0)) {
    std::vector<int> ts((size_t)b->tickets);
    for (size_t i = 0; i + 1 < start.size(); ++i)
      for (int64_t t = start[i]; t < start[i + 1]; ++t) ts[(size_t)t] = (int)i;
    BCUDA(cudaMalloc(&b->d_tslot, sizeof(int) * std::max<size_t>(ts.size(), 1)));
    if (!ts.empty()) BCUDA(cudaMemcpy(b->d_tslot, ts.data(), sizeof(int) * ts.size(), cudaMemcpyHostToDevice));
  }
  b->smem = std::max<size_t>(maxsmem, 16);
  BCUDA(cudaFuncSetAttribute(k_fft_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)std::max<size_t>(b->smem, 48 * 1024)));
  int dev = 0, sms = 148, per = 1;
  BCUDA(cudaGetDevice(&dev));
  BCUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_fft_batch<T>, kThreads, b->smem));
  b->grid = (unsigned)(sms * std::max(per, 1));
  char buf[256];
  snprintf(buf, sizeof(buf),
           "{\"transforms\":%d,\"slots\":%d,\"tiles\":%lld,\"lengths\":%zu,\"smem\":%zu,\"grid\":%u,"
           "\"alg_bytes\":%lld}",
           b->count, b->nslots, (long long)b->tickets, lens.size(), b->smem, b->grid,
           (long long)b->alg_bytes);
  b->desc = buf;
  return 0;
}

template <typename T>
int batch_launch(shafft_sm100_batch_s* b, int conj, double scale, cudaStream_t s) {
  using C = typename Vec2<T>::type;
  BCUDA(cudaMemsetAsync(b->d_ctl, 0, sizeof(int) * (4 + b->nslots), s));
  k_fft_batch<T><<<b->grid, kThreads, b->smem, s>>>(
      reinterpret_cast<const SlotDesc<C>*>(b->d_slots), b->d_start, b->d_tslot, b->nslots,
      reinterpret_cast<C* const*>(b->d_src), reinterpret_cast<C* const*>(b->d_dst), b->d_ctl + 4,
      reinterpret_cast<unsigned long long*>(b->d_ctl), b->d_ctl + 2, conj, scale, b->wait_limit);
  BCUDA(cudaGetLastError());
  return 0;
}

void batch_free(shafft_sm100_batch_s* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->d_tables);
  cudaFree(b->d_slots);
  cudaFree(b->d_start);
  if (b->d_tslot) cudaFree(b->d_tslot);
  cudaFree(b->d_ctl);
  cudaFree(b->d_src);
  cudaFree(b->d_dst);
}

}  // namespace

extern "C" {

int shafft_sm100_batch_create(shafft_sm100_batch* out, int count, const int* ndims,
                              const int64_t* dims, int precision, int flags) {
  if (!out || count < 1 || !ndims || !dims) return bfail(SHAFFT_SM100_EINVAL, "bad batch arguments");
  if (precision != 0 && precision != 1) return bfail(SHAFFT_SM100_EINVAL, "bad precision");
  *out = nullptr;
  auto* b = new (std::nothrow) shafft_sm100_batch_s();
  if (!b) return bfail(SHAFFT_SM100_EALLOC, "host allocation failed");
  b->precision = precision;
  b->count = count;
  b->ndims.assign(ndims, ndims + count);
  int64_t nd_total = 0;
  for (int i = 0; i < count; ++i) {
    if (ndims[i] < 1 || ndims[i] > 16) {
      delete b;
      return bfail(SHAFFT_SM100_EINVAL, "transform %d: ndim %d", i, ndims[i]);
    }
    nd_total += ndims[i];
  }
  b->dims.assign(dims, dims + nd_total);
  const int64_t* dp = dims;
  for (int i = 0; i < count; ++i) {
    int64_t n = 1;
    for (int a = 0; a < ndims[i]; ++a) {
      if (dp[a] < 1) {
        delete b;
        return bfail(SHAFFT_SM100_EINVAL, "transform %d: axis %d has length %lld", i, a,
                     (long long)dp[a]);
      }
      n *= dp[a];
    }
    dp += ndims[i];
    b->elements.push_back(n);
  }
  const int autotune = (flags & 1) ? 1 : 0;
  int rc = precision ? batch_build<double>(b, autotune) : batch_build<float>(b, autotune);
  if (rc) {
    batch_free(b);
    delete b;
    return rc;
  }
  *out = b;
  return 0;
}

int shafft_sm100_batch_destroy(shafft_sm100_batch b) {
  if (!b) return 0;
  batch_free(b);
  delete b;
  return 0;
}

int shafft_sm100_batch_execute(shafft_sm100_batch b, void* const* src, void* const* dst,
                               int direction, double scale, void* stream) {
  if (!b || !src || !dst) return bfail(SHAFFT_SM100_EINVAL, "null argument");
  if (direction != 0 && direction != 1) return bfail(SHAFFT_SM100_EINVAL, "bad direction");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool same_ptrs = (int)b->h_src.size() == b->count &&
                         std::equal(src, src + b->count, b->h_src.begin()) &&
                         std::equal(dst, dst + b->count, b->h_dst.begin());
  if (!same_ptrs) {
    b->h_src.assign(src, src + b->count);
    b->h_dst.assign(dst, dst + b->count);
    BCUDA(cudaMemcpyAsync(b->d_src, b->h_src.data(), sizeof(void*) * b->count,
                          cudaMemcpyHostToDevice, s));
    BCUDA(cudaMemcpyAsync(b->d_dst, b->h_dst.data(), sizeof(void*) * b->count,
                          cudaMemcpyHostToDevice, s));
    BCUDA(cudaStreamSynchronize(s));
  }
  // replay the captured graph (counter reset + the persistent launch) when
  // the call matches the captured one; otherwise capture a new graph
  if (!b->graph || b->graph_conj != direction || b->graph_scale != scale) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaStream_t cap = nullptr;
    BCUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    BCUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = b->precision ? batch_launch<double>(b, direction, scale, cap)
                          : batch_launch<float>(b, direction, scale, cap);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return bfail(SHAFFT_SM100_ECUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bfail(SHAFFT_SM100_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
    b->graph_conj = direction;
    b->graph_scale = scale;
    b->graph_stream = s;
  }
  BCUDA(cudaGraphLaunch(b->graph, s));
  return 0;
}

int shafft_sm100_batch_set_wait_limit(shafft_sm100_batch b, unsigned polls) {
  if (!b) return bfail(SHAFFT_SM100_EINVAL, "null batch");
  const unsigned limit = polls ? polls : kBatchSpinLimit;
  if (limit != b->wait_limit && b->graph) {  // the limit is a launch argument of the captured graph
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->wait_limit = limit;
  return 0;
}

int shafft_sm100_batch_status(shafft_sm100_batch b) {
  if (!b) return bfail(SHAFFT_SM100_EINVAL, "null batch");
  int flag = 0;
  BCUDA(cudaMemcpy(&flag, b->d_ctl + 2, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return bfail(SHAFFT_SM100_ECUDA, "batch: a wait for a previous pass timed out");
  return 0;
}

int64_t shafft_sm100_batch_bytes(shafft_sm100_batch b) { return b ? b->alg_bytes : 0; }

int shafft_sm100_batch_describe(shafft_sm100_batch b, char* buf, int buflen) {
  if (!b || !buf || buflen <= 0) return bfail(SHAFFT_SM100_EINVAL, "bad arguments");
  snprintf(buf, buflen, "%s", b->desc.c_str());
  return (int)b->desc.size() + 1 > buflen ? bfail(SHAFFT_SM100_EINVAL, "truncated") : 0;
}

}  // extern "C"
