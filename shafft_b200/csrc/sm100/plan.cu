// Planner, executor and C ABI of libshafft_sm100.so.
//
// The planner turns "C2C DFT over every axis of a row-major tensor" into a
// list of HBM passes (see pass.h).  Per axis of length L, inner stride I and
// outer count O:
//   * L == 1                       -> nothing;
//   * L smooth, fits one pass      -> one pass (row tile if I == 1, column
//                                     tile otherwise), in place;
//   * L smooth, too long           -> global decimation in frequency over
//                                     2 or 3 passes: pass s does DFTs of
//                                     length L_s at stride L/(L_0..L_s)*I and
//                                     multiplies by w_span^{j*k}; the last pass
//                                     undoes the digit reversal while storing
//                                     (out of place);
//   * L with a prime factor > 13   -> Bluestein: modulate by the chirp into
//                                     scratch rows of power-of-two length
//                                     M >= 2L-1, FFT_M, multiply by the
//                                     precomputed kernel spectrum, FFT_M,
//                                     demodulate.
// This replaces the reference's per-axis-group hipFFT plans
// (src/cpp/fft/hipfft_method/fftnd_method.cpp:47-61, 73-158, 162-351), its
// gpuTT transpose path (src/cpp/fft/hipfft_method/nd/transpose_fftnd.cpp)
// and its Bluestein executor
// (src/cpp/fft/hipfft_method/1d/fft1d_bluestein_executor.hip:249-356).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../../include/shafft_sm100.h"
#include "launch.h"
#include "pass.h"

namespace shafft_sm100 {

static thread_local int g_last_cuda = 0;
static thread_local char g_last_msg[512] = "";

static int set_err(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
static int set_err(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_msg, sizeof(g_last_msg), fmt, ap);
  va_end(ap);
  return code;
}

int report_error(int code, const char* msg) {
  snprintf(g_last_msg, sizeof(g_last_msg), "%s", msg);
  return code;
}

#define CUDA_TRY(expr)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      g_last_cuda = (int)e_;                                                             \
      return set_err(SHAFFT_SM100_ECUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                                \
    }                                                                                    \
  } while (0)

enum StepKind : int { ST_PASS = 0, ST_BS_MOD, ST_BS_MULH, ST_BS_DEMOD, ST_COPY, ST_PLANE };
enum BufId : int { BUF_SRC = 0, BUF_DST = 1, BUF_S0 = 2, BUF_S1 = 3 };

static int other_buf(int b) {
  switch (b) {
    case BUF_SRC: return BUF_DST;
    case BUF_DST: return BUF_SRC;
    case BUF_S0: return BUF_S1;
    default: return BUF_S0;
  }
}

static const char* buf_name(int b) {
  static const char* n[] = {"src", "dst", "s0", "s1"};
  return n[b & 3];
}

struct Step {
  int kind = ST_PASS;
  PassGeom g{};
  int in_buf = BUF_SRC, out_buf = BUF_DST;
  int tabL = -1, tabN = -1, tabB = -1;
  int64_t bsL = 0, bsM = 0, bsI = 1, total = 0;
  size_t smem = 0;
  int fast = 0;      // 1: specialised k_fft_fast pass (compile-time L)
  int fast_row = 0;  // specialised pass reads row tiles (transposing)
  int tc = 0;        // 1: tensor-core pass (tcgen05 split-FP16 DFT GEMM, L <= 64)
  // ST_PLANE: g = X phase (src -> mid), g2 = Y phase (mid -> out)
  PassGeom g2{};
  int mid_buf = BUF_DST;
  int lag = 4;
  int64_t planes = 0;
  size_t off_ctl = 0;  // control words (4 + planes ints) in the plan's table blob
  // ST_PLANE with cluster = 1: the two axes of each L x L plane in one pass
  // of k_fft_plane_cluster (a thread-block cluster holds the plane in
  // distributed shared memory); in_buf -> out_buf, planes of L*L elements
  int cluster = 0;
};

// NVTX label of a step's launch (static strings: nothing is formatted on
// the execute path)
const char* step_label(const Step& st) {
  if (st.kind == ST_PLANE)
    return st.cluster ? "shafft_sm100 plane pass (two axes, cluster)" : "shafft_sm100 plane pass (two axes)";
  if (st.kind == ST_COPY) return "shafft_sm100 copy";
  if (st.kind != ST_PASS) return "shafft_sm100 bluestein element-wise step";
  if (st.tc) return "shafft_sm100 tensor-core pass";
  if (st.fast) return st.fast_row ? "shafft_sm100 pass (row tiles, transposing)" : "shafft_sm100 pass (column tiles)";
  return "shafft_sm100 generic pass";
}

struct LTable {
  int L;
  size_t off_tw, off_p2k, off_k2p;
  size_t off_tcB = 0, tc_bytes = 0;  // split DFT matrix of tensor-core passes
};
struct NTable {
  int64_t N;
  int shift;
  int64_t mask, nhi, nlo;
  size_t off_hi, off_lo;
};
struct BTable {
  int64_t L, M;
  size_t off_chirp, off_H;
  std::vector<Step> hsteps;  // FFT_M of the kernel sequence (S0 -> result buf)
  int hresult_buf;
};

struct Limits {
  int max_row;   // longest row-tile pass
  int max_col;   // longest column-tile pass
  int e_target;  // tile elements aimed at (64 KiB of complex data)
  int w_col;     // widest column tile
};

static Limits limits_for(int precision) {
  if (precision == 0) return Limits{4096, 2048, 8192, 16};
  return Limits{4096, 2048, 4096, 8};
}

// longest non-smooth length handled by a direct-DFT pass
constexpr int64_t kDirectMax = 1024;
// longest direct-DFT pass (SHAFFT_SM100_DIRECT_MAX overrides, up to 1024)
static int64_t direct_max() {
  if (const char* e = getenv("SHAFFT_SM100_DIRECT_MAX")) {
    const int64_t v = atoll(e);
    if (v >= 0 && v <= 1024) return v;
  }
  return kDirectMax;
}

static bool is_smooth(int64_t L) {
  const int64_t primes[] = {2, 3, 5, 7, 11, 13};
  for (int64_t p : primes)
    while (L % p == 0) L /= p;
  return L == 1;
}

static int pow2floor(int64_t x) {
  int p = 1;
  while ((int64_t)p * 2 <= x && p < (1 << 30)) p *= 2;
  return p;
}
static int pow2ceil(int64_t x) {
  int p = 1;
  while (p < x && p < (1 << 30)) p *= 2;
  return p;
}

struct Planner {
  int precision;
  Limits lim;
  size_t elem;
  std::vector<LTable> ltabs;
  std::vector<NTable> ntabs;
  std::vector<BTable> btabs;
  size_t table_bytes = 0;
  int64_t scratch_elems = 0;

  // Planning choices that measurements decide (SHAFFT_SM100_PLAN_MEASURE
  // times them per shape; the defaults are the measured-best rules):
  //   balanced  multi-pass splits as balanced as possible (default for
  //             complex64) instead of the largest last factor
  //   widen     narrower generic tiles for passes with few tiles
  int balanced = -1;  // -1: by precision
  int widen = 1;
  // tensor-core planning: every pass of length <= 64 is a tcgen05 pass
  int tc_mode = 0;
  bool cur_tc = false;  // set while the passes being built are tensor-core passes
  size_t off_tcerr = 0;

  explicit Planner(int prec, int flags = 0)
      : precision(prec), lim(limits_for(prec)), elem(prec ? 16 : 8) {
    // 1: every pass on the tensor cores; 2: only axes with a prime factor
    // above 13 (where the plain path would run O(L^2) direct DFTs)
    tc_mode = prec != 0 ? 0
              : (flags & SHAFFT_SM100_PLAN_TENSOR_CORE) ? 1
              : (flags & SHAFFT_SM100_PLAN_TC_PRIME_AXES) ? 2 : 0;
    // device error word of passes with bounded waits (tensor-core and
    // bulk-copy column passes); 0 = ok
    off_tcerr = alloc(16);
    if (const char* e = getenv("SHAFFT_SM100_PLANE")) plane_enabled = atoi(e) != 0;
    if (const char* e = getenv("SHAFFT_SM100_PLANE_CLUSTER")) plane_cluster_enabled = atoi(e) != 0;
    if (const char* e = getenv("SHAFFT_SM100_FLOW_LAG")) flow_lag = std::max(1, atoi(e));
    if (const char* e = getenv("SHAFFT_SM100_ROTATE")) rotate_enabled = atoi(e) != 0;
  }

  // specialised-pass eligibility: length, tile width and 16-byte alignment
  int fast_w() const { return precision ? 8 : 16; }
  int vw() const { return precision ? 1 : 2; }
  bool fast_len(int64_t L) const {
    if (L > 1 << 20) return false;
    return precision ? Launch<double>::fast_supported((int)L) : Launch<float>::fast_supported((int)L);
  }
  bool fast_geom(const PassGeom& g, bool in_row) const {
    const int v = vw();
    if (g.ext[0] % fast_w() != 0) return false;
    if (g.sout[0] != 1) return false;
    if (!in_row && g.sin[0] != 1) return false;
    if (in_row && g.sn_in != 1) return false;
    if (g.sk_out % v) return false;
    if (!in_row && g.sn_in % v) return false;
    for (int d = 1; d < 4; ++d)
      if (g.sout[d] % v || (!in_row && g.sin[d] % v)) return false;
    return true;
  }
  // turn a planned generic pass into a specialised one when it qualifies
  void try_fast(Step& st) {
    if (cur_tc) return mark_tc(st);
    PassGeom& g = st.g;
    if (!fast_len(g.L) || g.tw_mode == TW_PRE) return;
    const bool in_row = (g.sn_in == 1);
    if (!fast_geom(g, in_row)) return;
    if (in_row && st.in_buf == st.out_buf) return;  // transposing pass must be out of place
    st.fast = 1;
    st.fast_row = in_row ? 1 : 0;
    finish_geom(st, fast_w());
    st.smem = (size_t)g.L * 128;
  }

  // Generic passes of small transforms can have too few tiles to fill the
  // GPU: halve the tile width (down to 2) while a pass has fewer tiles than
  // one wave of two CTAs per SM.  Measured on B200 (fwd+bwd): 121,500
  // 0.079 -> 0.035 ms, 3^11 0.083 -> 0.045 ms, 97x64 0.062 -> 0.030 ms;
  // passes that already have a few hundred tiles lose from narrower tiles
  // (105^3, 1,488,375), so they are left alone.
  void widen_grid(Step& st) {
    if (!widen || st.fast || st.tc || st.kind != ST_PASS) return;
    const int64_t want = 2 * 148;
    while (st.g.W > 2 && st.g.ntiles < want) finish_geom(st, st.g.W / 2);
  }

  void mark_tc(Step& st) {
    st.tc = 1;
    st.fast = 0;
    st.smem = tc_smem_bytes(st.g.L);
    LTable& lt = ltabs[st.tabL];
    if (!lt.tc_bytes) {
      lt.tc_bytes = tc_table_bytes(st.g.L);
      lt.off_tcB = alloc(lt.tc_bytes);
    }
  }

  size_t alloc(size_t bytes) {
    size_t off = (table_bytes + 255) & ~size_t(255);
    table_bytes = off + bytes;
    return off;
  }

  int ltab(int L) {
    for (size_t i = 0; i < ltabs.size(); ++i)
      if (ltabs[i].L == L) return (int)i;
    LTable t;
    t.L = L;
    t.off_tw = alloc(elem * L);
    t.off_p2k = alloc(2 * L);
    t.off_k2p = alloc(2 * L);
    ltabs.push_back(t);
    return (int)ltabs.size() - 1;
  }

  int ntab(int64_t N) {
    for (size_t i = 0; i < ntabs.size(); ++i)
      if (ntabs[i].N == N) return (int)i;
    NTable t;
    t.N = N;
    int lg = 0;
    while ((int64_t(1) << lg) < N) ++lg;
    t.shift = (lg + 1) / 2;
    t.mask = (int64_t(1) << t.shift) - 1;
    t.nlo = int64_t(1) << t.shift;
    t.nhi = (N + t.nlo - 1) / t.nlo + 1;
    t.off_hi = alloc(elem * t.nhi);
    t.off_lo = alloc(elem * t.nlo);
    ntabs.push_back(t);
    return (int)ntabs.size() - 1;
  }

  // radix stages of a pass of length L; nst = 0 (direct DFT) when L has a
  // prime factor above 13
  void fill_radix(PassGeom& g, int L) {
    RadixPlan rp = radix_plan(L);
    g.L = L;
    g.nst = rp.n > 0 ? rp.n : 0;
    for (int s = 0; s < g.nst; ++s) g.rad[s] = rp.r[s];
  }

  void finish_geom(Step& st, int W) {
    PassGeom& g = st.g;
    g.W = W;
    g.logW = 0;
    while ((1 << g.logW) < W) ++g.logW;
    for (int d = 0; d < 4; ++d)
      if (g.ext[d] < 1) g.ext[d] = 1;
    g.tiles_w = (g.ext[0] + W - 1) / W;
    g.ntiles = g.tiles_w * g.ext[1] * g.ext[2] * g.ext[3];
    g.in_row = (g.sn_in == 1) ? 1 : 0;
    g.out_row = (g.sk_out == 1) ? 1 : 0;
    g.pitch = generic_pitch(W, g.in_row != 0);
    g.scale = 1.0;
    st.smem = (size_t)g.L * (size_t)g.pitch * elem;
    st.tabL = ltab(g.L);
  }

  int col_width(int L, int64_t I) const {
    int w = lim.e_target / L;
    if (w < 1) w = 1;
    w = std::min(w, lim.w_col);
    w = pow2floor(w);
    w = std::min(w, pow2ceil(I));
    return std::max(w, 1);
  }

  // one pass over axis (O, L, I): in_buf -> out_buf (may be equal)
  void single_pass(std::vector<Step>& out, int64_t O, int L, int64_t I, int in_buf, int out_buf) {
    Step st;
    st.kind = ST_PASS;
    st.in_buf = in_buf;
    st.out_buf = out_buf;
    fill_radix(st.g, L);
    PassGeom& g = st.g;
    if (I == 1) {
      int W = pow2floor(std::max<int64_t>(1, std::min<int64_t>(O, lim.e_target / L)));
      W = std::min(W, 32);
      g.ext[0] = O;
      g.sin[0] = g.sout[0] = L;
      g.ext[1] = g.ext[2] = g.ext[3] = 1;
      g.sn_in = g.sk_out = 1;
      finish_geom(st, W);
      if (cur_tc) mark_tc(st);
      widen_grid(st);
    } else {
      int W = col_width(L, I);
      g.ext[0] = I;
      g.sin[0] = g.sout[0] = 1;
      g.ext[1] = O;
      g.sin[1] = g.sout[1] = (int64_t)L * I;
      g.ext[2] = g.ext[3] = 1;
      g.sn_in = g.sk_out = I;
      finish_geom(st, W);
      try_fast(st);
      widen_grid(st);
    }
    out.push_back(st);
  }

  bool plane_len(int64_t L) const {
    if (L > 1 << 20) return false;
    return precision ? Launch<double>::plane_supported((int)L) : Launch<float>::plane_supported((int)L);
  }

  // The last two axes of a stack of O square L x L planes in one HBM pass
  // (k_fft_plane): buf -> (mid = other(buf)) -> buf.
  bool plane_step(std::vector<Step>& out, int64_t O, int64_t L, int buf) {
    if (!plane_enabled || !plane_len(L) || L % fast_w() || O < 16 || O > (1 << 24)) return false;
    std::vector<Step> tmp;
    if (!transposed_pair(tmp, O, L, L, buf, other_buf(buf), buf)) return false;
    Step st;
    st.kind = ST_PLANE;
    st.g = tmp[0].g;
    st.g2 = tmp[1].g;
    st.in_buf = buf;
    st.mid_buf = other_buf(buf);
    st.out_buf = buf;
    st.tabL = tmp[0].tabL;
    st.smem = (size_t)L * 128;
    st.planes = O;
    st.lag = flow_lag;
    st.off_ctl = alloc(sizeof(int) * (size_t)(4 + O));
    out.push_back(st);
    return true;
  }
  int plane_enabled = 0;  // SHAFFT_SM100_PLANE=1 turns the fused plane pass on (slower so far)

  // The last two axes of a stack of O L x L planes in one pass of the cluster
  // plane kernel, in place on buf (the parity fix may turn it out of place).
  bool plane_cluster_step(std::vector<Step>& out, int64_t O, int64_t L, int buf) {
    if (!plane_cluster_enabled || tc_mode == 1 || !plane_cluster_len(precision, L)) return false;
    Step st;
    st.kind = ST_PLANE;
    st.cluster = 1;
    st.in_buf = st.mid_buf = st.out_buf = buf;
    fill_radix(st.g, (int)L);
    st.g.ext[0] = st.g.ext[1] = st.g.ext[2] = st.g.ext[3] = 1;
    st.tabL = ltab((int)L);
    st.smem = plane_cluster_smem();
    st.planes = O;
    out.push_back(st);
    return true;
  }
  // SHAFFT_SM100_PLANE_CLUSTER=0 turns the cluster plane pass off; plan
  // creation also turns it off on a device that cannot co-schedule the
  // clusters
  int plane_cluster_enabled = 0;
  int flow_lag = 4;       // SHAFFT_SM100_FLOW_LAG: planes between an X tile and its Y tile

  // The last two axes (A = rows, Lr = contiguous) as two transposing passes:
  // rows of Lr -> [o][kL][a] in `mid`, then rows of A -> [o][ka][kL] in
  // out_buf.  Both passes read row tiles and store column tiles.
  bool transposed_pair(std::vector<Step>& out, int64_t O, int64_t A, int64_t Lr, int in_buf,
                       int mid_buf, int out_buf) {
    if (!fast_len(A) || !fast_len(Lr) || A % fast_w() || Lr % fast_w()) return false;
    Step s1;
    s1.kind = ST_PASS;
    s1.in_buf = in_buf;
    s1.out_buf = mid_buf;
    fill_radix(s1.g, (int)Lr);
    s1.g.ext[0] = A;  s1.g.sin[0] = Lr;  s1.g.sout[0] = 1;
    s1.g.ext[1] = O;  s1.g.sin[1] = s1.g.sout[1] = A * Lr;
    s1.g.ext[2] = s1.g.ext[3] = 1;
    s1.g.sn_in = 1;
    s1.g.sk_out = A;
    finish_geom(s1, fast_w());
    Step s2;
    s2.kind = ST_PASS;
    s2.in_buf = mid_buf;
    s2.out_buf = out_buf;
    fill_radix(s2.g, (int)A);
    s2.g.ext[0] = Lr;  s2.g.sin[0] = A;  s2.g.sout[0] = 1;
    s2.g.ext[1] = O;  s2.g.sin[1] = s2.g.sout[1] = A * Lr;
    s2.g.ext[2] = s2.g.ext[3] = 1;
    s2.g.sn_in = 1;
    s2.g.sk_out = Lr;
    finish_geom(s2, fast_w());
    try_fast(s1);
    try_fast(s2);
    if (!s1.fast || !s2.fast) return false;
    out.push_back(s1);
    out.push_back(s2);
    return true;
  }

  // choose 2- or 3-factor split of a smooth L; returns empty if impossible
  std::vector<int> split(int64_t L, int64_t I) const {
    // SHAFFT_SM100_FACTORS="a,b[,c]": factor list for an axis of length a*b*c
    // (planning experiments); ignored for any other length
    if (const char* e = getenv("SHAFFT_SM100_FACTORS")) {
      std::vector<int> f;
      int64_t prod = 1;
      for (const char* q = e; *q;) {
        const long v = strtol(q, const_cast<char**>(&q), 10);
        if (v < 2) break;
        f.push_back((int)v);
        prod *= v;
        if (*q == ',') ++q;
      }
      if (prod == L && f.size() >= 2 && f.size() <= 3) return f;
    }
    // Prefer factors that all have a specialised pass, the fewest passes, and
    // for complex64 among those the most balanced split (largest smallest
    // factor; ties to the larger last factor).  Balanced splits keep tiles small enough for
    // several CTAs per SM: measured on B200, 2^24 = 256*256*256 runs 17%
    // faster than 16*1024*1024.
    {
      const int64_t fl[] = {1024, 512, 256, 128, 64, 32, 16};
      std::vector<int> best2, best3;
      int64_t m2 = 0, m3 = 0;
      for (int64_t d : fl) {
        if (L % d || !fast_len(d)) continue;
        const int64_t c = L / d;
        // complex128 (tiles twice the bytes): the largest last factor wins
        // instead (2^24 = 64*512*512: 0.78 ms vs 0.87 ms for 256^3)
        const bool first_only = balanced < 0 ? precision != 0 : balanced == 0;
        if (fast_len(c) && c >= 16 && std::min(c, d) > m2 && !(first_only && m2 > 0)) {
          m2 = std::min(c, d);
          best2 = {(int)c, (int)d};
        }
        for (int64_t f : fl) {
          if (c % f || !fast_len(f) || !fast_len(c / f) || c / f < 16) continue;
          const int64_t mn = std::min(std::min(c / f, f), d);
          if (mn > m3 && !(first_only && m3 > 0)) {
            m3 = mn;
            best3 = {(int)(c / f), (int)f, (int)d};
          }
        }
      }
      if (!best2.empty()) return best2;
      if (!best3.empty()) return best3;
    }
    const int max_last = (I == 1) ? lim.max_row : lim.max_col;
    std::vector<int> best;
    // 2 factors, as balanced as the pass limits allow (smaller one first):
    // 1,488,375 = 1215*1225 measured 17% faster than 375*3969
    {
      int64_t bm = 0;
      for (int64_t d = std::min<int64_t>(L, max_last); d >= 2; --d) {
        if (L % d) continue;
        const int64_t c = L / d;
        if (c < 2 || c > lim.max_col || std::min(c, d) <= bm) continue;
        bm = std::min(c, d);
        best = {(int)c, (int)d};
        if (balanced == 0) break;  // the largest last factor that fits
      }
    }
    if (!best.empty()) return best;
    for (int64_t d = std::min<int64_t>(L, max_last); d >= 2; --d) {
      if (L % d) continue;
      int64_t c = L / d;
      // split c into two column factors as balanced as possible
      int64_t bestf = -1;
      for (int64_t f = 2; f * f <= c; ++f)
        if (c % f == 0 && f <= lim.max_col && c / f <= lim.max_col) bestf = f;
      if (bestf > 0) return {(int)(c / bestf), (int)bestf, (int)d};
    }
    return {};
  }

  // global decimation-in-frequency over the factors Ls
  void multi_pass(std::vector<Step>& out, int64_t O, int64_t L, int64_t I, const std::vector<int>& Ls,
                  int in_buf, int out_buf) {
    const int S = (int)Ls.size();
    int64_t span = L;
    // in-place passes
    for (int s = 0; s < S - 1; ++s) {
      const int R = Ls[s];
      const int64_t m = span / R;
      Step st;
      st.kind = ST_PASS;
      st.in_buf = (s == 0) ? in_buf : out_buf;
      st.out_buf = out_buf;
      fill_radix(st.g, R);
      PassGeom& g = st.g;
      g.sn_in = g.sk_out = m * I;
      int W;
      if (I > 1) {
        g.ext[0] = I;  g.sin[0] = g.sout[0] = 1;
        g.ext[1] = m;  g.sin[1] = g.sout[1] = I;
        g.ext[2] = L / span;  g.sin[2] = g.sout[2] = span * I;
        g.ext[3] = O;  g.sin[3] = g.sout[3] = L * I;
        g.tw_dim = 1;
        W = col_width(R, I);
      } else {
        g.ext[0] = m;  g.sin[0] = g.sout[0] = 1;
        g.ext[1] = L / span;  g.sin[1] = g.sout[1] = span;
        g.ext[2] = O;  g.sin[2] = g.sout[2] = L;
        g.ext[3] = 1;  g.sin[3] = g.sout[3] = 0;
        g.tw_dim = 0;
        W = col_width(R, m);
      }
      g.tw_mode = TW_POST;
      st.tabN = ntab(span);
      finish_geom(st, W);
      try_fast(st);
      widen_grid(st);
      out.push_back(st);
      span = m;
    }
    // last pass: undo digit reversal while storing
    {
      const int R = Ls[S - 1];
      Step st;
      st.kind = ST_PASS;
      st.in_buf = (S == 1) ? in_buf : out_buf;
      st.out_buf = other_buf(st.in_buf);
      fill_radix(st.g, R);
      PassGeom& g = st.g;
      g.sn_in = I;
      g.sk_out = (L / R) * I;
      // digit t: input stride m_t*I, output stride (L_0..L_{t-1})*I
      int64_t din[3] = {0, 0, 0}, dout[3] = {0, 0, 0}, dext[3] = {1, 1, 1};
      int64_t prod = 1;
      for (int t = 0; t < S - 1; ++t) {
        prod *= Ls[t];
        dext[t] = Ls[t];
        din[t] = (L / prod) * I;
        dout[t] = (prod / Ls[t]) * I;
      }
      int W;
      if (I > 1) {
        g.ext[0] = I;  g.sin[0] = g.sout[0] = 1;
        g.ext[1] = dext[0];  g.sin[1] = din[0];  g.sout[1] = dout[0];
        g.ext[2] = dext[1];  g.sin[2] = din[1];  g.sout[2] = dout[1];
        g.ext[3] = O;  g.sin[3] = g.sout[3] = L * I;
        W = col_width(R, I);
      } else if (S == 4) {
        g.ext[0] = dext[0];  g.sin[0] = din[0];  g.sout[0] = dout[0];
        g.ext[1] = dext[1];  g.sin[1] = din[1];  g.sout[1] = dout[1];
        g.ext[2] = dext[2];  g.sin[2] = din[2];  g.sout[2] = dout[2];
        g.ext[3] = O;  g.sin[3] = g.sout[3] = L;
        W = 1;
      } else {
        g.ext[0] = dext[0];  g.sin[0] = din[0];  g.sout[0] = dout[0];
        g.ext[1] = dext[1];  g.sin[1] = din[1];  g.sout[1] = dout[1];
        g.ext[2] = O;  g.sin[2] = g.sout[2] = L;
        g.ext[3] = 1;  g.sin[3] = g.sout[3] = 0;
        // row tile in, column tile out: W rows of R contiguous inputs
        W = pow2floor(std::max<int64_t>(1, std::min<int64_t>(dext[0], lim.e_target / R)));
        W = std::min(W, lim.w_col);
      }
      finish_geom(st, W);
      try_fast(st);
      widen_grid(st);
      out.push_back(st);
    }
  }

  int btab(int64_t L, int64_t M) {
    for (size_t i = 0; i < btabs.size(); ++i)
      if (btabs[i].L == L && btabs[i].M == M) return (int)i;
    BTable t;
    t.L = L;
    t.M = M;
    t.off_chirp = alloc(elem * L);
    t.off_H = alloc(elem * M);
    scratch_elems = std::max(scratch_elems, M);
    // the kernel spectrum FFT_M(h): plan it on scratch S0 -> ...
    int cur = BUF_S0;
    int rc = axis(t.hsteps, 1, M, 1, cur, false, /*in_bluestein=*/true);
    (void)rc;
    t.hresult_buf = cur;
    btabs.push_back(t);
    return (int)btabs.size() - 1;
  }

  // Plan one axis; `cur` holds the data on entry and on exit.
  // Factor L into S <= max_s factors, each in 2..64, as balanced as possible
  // (largest smallest factor); empty if L has a prime factor above 64 or
  // needs more factors.
  static std::vector<int> tc_split(int64_t L, int max_s) {
    std::vector<int> best;
    for (int S = 2; S <= max_s && best.empty(); ++S) {
      std::vector<int> cur;
      int best_min = 0;
      // depth-first over non-increasing factor sequences
      std::function<void(int64_t, int)> rec = [&](int64_t rem, int hi) {
        const int k = (int)cur.size();
        if (k == S - 1) {
          if (rem >= 2 && rem <= hi) {
            cur.push_back((int)rem);
            const int mn = *std::min_element(cur.begin(), cur.end());
            if (mn > best_min) {
              best_min = mn;
              best = cur;
            }
            cur.pop_back();
          }
          return;
        }
        for (int f = hi; f >= 2; --f) {
          if (rem % f) continue;
          cur.push_back(f);
          rec(rem / f, f);
          cur.pop_back();
        }
      };
      rec(L, 64);
    }
    // multi_pass runs factors first-to-last; the last one is the row pass
    std::reverse(best.begin(), best.end());
    return best;
  }

  // Tensor-core route for one axis; false when the axis needs the plain path.
  bool tc_axis(std::vector<Step>& out, int64_t O, int64_t L, int64_t I, int& cur, bool force_oop) {
    if (!tc_mode) return false;
    if (tc_mode == 2 && is_smooth(L)) return false;  // smooth axes keep the plain passes
    if (L <= 64) {
      cur_tc = true;
      const int ob = force_oop ? other_buf(cur) : cur;
      single_pass(out, O, (int)L, I, cur, ob);
      cur_tc = false;
      cur = ob;
      return true;
    }
    std::vector<int> f = tc_split(L, I == 1 ? 4 : 3);
    if (f.empty()) return false;
    cur_tc = true;
    const int x = force_oop ? other_buf(cur) : cur;
    multi_pass(out, O, L, I, f, cur, x);
    cur_tc = false;
    cur = out.back().out_buf;
    return true;
  }

  int axis(std::vector<Step>& out, int64_t O, int64_t L, int64_t I, int& cur, bool force_oop,
           bool in_bluestein) {
    if (L == 1) return 0;
    if (tc_axis(out, O, L, I, cur, force_oop)) return 0;
    const int max_one = (I == 1) ? lim.max_row : lim.max_col;
    if (is_smooth(L) && L <= max_one) {
      int ob = force_oop ? other_buf(cur) : cur;
      single_pass(out, O, (int)L, I, cur, ob);
      cur = ob;
      return 0;
    }
    if (is_smooth(L)) {
      std::vector<int> f = split(L, I);
      if (!f.empty()) {
        // the last pass is out of place: it lands in other(x) where x is the
        // buffer the in-place passes used
        const int x = force_oop ? other_buf(cur) : cur;
        multi_pass(out, O, L, I, f, cur, x);
        cur = out.back().out_buf;
        return 0;
      }
    }
    if (in_bluestein) return SHAFFT_SM100_ENOTSUP;
    // short lengths with a large prime factor: one direct-DFT pass instead
    // of the five Bluestein steps.  The paired direct DFT costs about L / 4
    // multiply-adds per point, Bluestein a few passes over M >= 2L - 1
    // points; measured on B200 (rows of 131 .. 1021 points) the direct pass
    // wins while L^2 <= 128 M, which holds for every L up to 362 and for
    // none above (from 513 on, M = 2048 pads too little to pay).
    int64_t Mb = 1;
    while (Mb < 2 * L - 1) Mb <<= 1;
    if (L <= direct_max() && L * L <= 128 * Mb) {
      int ob = force_oop ? other_buf(cur) : cur;
      single_pass(out, O, (int)L, I, cur, ob);
      cur = ob;
      return 0;
    }
    // Bluestein
    int64_t M = 1;
    while (M < 2 * L - 1) M <<= 1;
    const int64_t B = O * I;
    const int bt = btab(L, M);
    scratch_elems = std::max(scratch_elems, B * M);
    Step mod;
    mod.kind = ST_BS_MOD;
    mod.in_buf = cur;
    mod.out_buf = BUF_S0;
    mod.tabB = bt;
    mod.bsL = L;
    mod.bsM = M;
    mod.bsI = I;
    mod.total = B * M;
    out.push_back(mod);
    int sc = BUF_S0;
    int rc = axis(out, B, M, 1, sc, false, true);
    if (rc) return rc;
    Step mul;
    mul.kind = ST_BS_MULH;
    mul.in_buf = mul.out_buf = sc;
    mul.tabB = bt;
    mul.bsM = M;
    mul.total = B * M;
    out.push_back(mul);
    rc = axis(out, B, M, 1, sc, false, true);
    if (rc) return rc;
    Step dem;
    dem.kind = ST_BS_DEMOD;
    dem.in_buf = sc;
    dem.out_buf = force_oop ? other_buf(cur) : cur;
    dem.tabB = bt;
    dem.bsL = L;
    dem.bsM = M;
    dem.bsI = I;
    dem.total = B * L;
    out.push_back(dem);
    cur = dem.out_buf;
    return 0;
  }

  // Rotation chain for an odd number (>= 3) of non-trivial axes: each pass
  // transforms the contiguous axis (row tiles) and stores it as the slowest
  // index (column tiles), so after one pass per axis the layout is natural
  // again and every pass is a transposing pass; src -> dst -> ... -> dst.
  bool rotation_chain(std::vector<Step>& out, int ndim, const int64_t* dims) {
    std::vector<int64_t> ax;
    int64_t N = 1;
    for (int a = 0; a < ndim; ++a)
      if (dims[a] > 1) {
        ax.push_back(dims[a]);
        N *= dims[a];
      }
    if (ax.size() < 3 || ax.size() % 2 == 0) return false;
    std::vector<Step> tmp;
    int cur = BUF_SRC;
    for (int i = (int)ax.size() - 1; i >= 0; --i) {
      const int64_t L = ax[i];
      if (!fast_len(L) || (N / L) % fast_w()) return false;
      Step st;
      st.kind = ST_PASS;
      st.in_buf = cur;
      st.out_buf = other_buf(cur);
      fill_radix(st.g, (int)L);
      st.g.ext[0] = N / L;  st.g.sin[0] = L;  st.g.sout[0] = 1;
      st.g.sn_in = 1;
      st.g.sk_out = N / L;
      finish_geom(st, fast_w());
      try_fast(st);
      if (!st.fast) return false;
      tmp.push_back(st);
      cur = other_buf(cur);
    }
    out = tmp;
    return true;
  }
  int rotate_enabled = 0;  // SHAFFT_SM100_ROTATE=1: rotation chain for 3-D and odd-rank tensors

  // axes to transform (bit a = axis a); the others are batch axes
  uint64_t axes_mask = ~0ull;
  // a plan that loads an exchange's block layout: axes in increasing order,
  // one pass each (no transposing pair), with the first in-place step made
  // the out-of-place one, so that the first step can take the load map
  int load_first = 0;

  // SHAFFT_SM100_BS_FUSE=0 keeps Bluestein's element-wise steps as launches
  // of their own (for comparisons); by default they are fused into the
  // neighbouring specialised passes
  static bool bs_fuse_enabled() {
    const char* e = getenv("SHAFFT_SM100_BS_FUSE");
    return !(e && atoi(e) == 0);
  }

  // Fold Bluestein's element-wise steps into the specialised passes next to
  // them (rows of x with unit stride only): modulate into the loads of the
  // first pass of the forward convolution FFT when that pass reads column
  // tiles, the spectrum multiply into the stores of that FFT's last pass,
  // the demodulate (with the normalisation and output conjugation) into the
  // stores of the inverse FFT's last pass.  The same operations in the same
  // order as the unfused steps (results agree to rounding: the compiler may
  // contract them into fused multiply-adds differently in the two kernels).
  // Complex64 only: measured on B200, FFT1D 1,000,003 fwd+bwd went 0.141 ->
  // 0.123 ms fused, while complex128 went 0.296 -> 0.306 ms (its first
  // convolution pass is 16 points long, where the element-wise loads cost
  // more than the modulate kernel they replace).
  void fuse_bluestein(std::vector<Step>& out) {
    if (!bs_fuse_enabled() || precision != 0) return;
    auto fast_pass = [](const Step& st) { return st.kind == ST_PASS && st.fast && !st.tc; };
    auto logm = [](int64_t M) {
      int l = 0;
      while ((int64_t(1) << l) < M) ++l;
      return l;
    };
    for (size_t i = 0; i < out.size(); ++i) {
      Step& st = out[i];
      if (st.kind == ST_BS_MOD && st.bsI == 1 && i + 1 < out.size()) {
        Step& nx = out[i + 1];
        if (fast_pass(nx) && !nx.fast_row && nx.in_buf == st.out_buf && !nx.g.bs_mode) {
          nx.in_buf = st.in_buf;
          nx.g.bs_mode |= BS_LOAD_MOD;
          nx.g.bs_logM = logm(st.bsM);
          nx.g.bs_L = st.bsL;
          nx.tabB = st.tabB;
          out.erase(out.begin() + i);
          --i;
        }
      } else if (st.kind == ST_BS_MULH && i > 0) {
        Step& pv = out[i - 1];
        if (fast_pass(pv) && pv.out_buf == st.in_buf && st.in_buf == st.out_buf &&
            !(pv.g.bs_mode & (BS_STORE_MULH | BS_STORE_DEMOD)) && (pv.tabB < 0 || pv.tabB == st.tabB)) {
          pv.g.bs_mode |= BS_STORE_MULH;
          pv.g.bs_logM = logm(st.bsM);
          pv.tabB = st.tabB;
          out.erase(out.begin() + i);
          --i;
        }
      } else if (st.kind == ST_BS_DEMOD && st.bsI == 1 && i > 0) {
        Step& pv = out[i - 1];
        if (fast_pass(pv) && pv.out_buf == st.in_buf &&
            !(pv.g.bs_mode & (BS_STORE_MULH | BS_STORE_DEMOD)) && (pv.tabB < 0 || pv.tabB == st.tabB)) {
          pv.out_buf = st.out_buf;
          pv.g.bs_mode |= BS_STORE_DEMOD;
          pv.g.bs_logM = logm(st.bsM);
          pv.g.bs_L = st.bsL;
          pv.tabB = st.tabB;
          out.erase(out.begin() + i);
          --i;
        }
      }
    }
  }

  int plan_nd(std::vector<Step>& out, int ndim, const int64_t* dims) {
    const int rc = plan_nd_steps(out, ndim, dims);
    if (!rc) fuse_bluestein(out);
    return rc;
  }

  int plan_nd_steps(std::vector<Step>& out, int ndim, const int64_t* dims) {
    out.clear();
    auto on = [&](int a) { return dims[a] > 1 && ((axes_mask >> a) & 1ull); };
    const bool all_axes = (ndim >= 64) || ((~axes_mask) & ((1ull << ndim) - 1)) == 0;
    if (rotate_enabled && !tc_mode && all_axes && rotation_chain(out, ndim, dims)) return 0;
    int cur = BUF_SRC;
    int a = ndim - 1;
    if (load_first) {
      for (int b = 0; b < ndim; ++b) {
        int64_t I = 1, O = 1;
        for (int c = b + 1; c < ndim; ++c) I *= dims[c];
        for (int c = 0; c < b; ++c) O *= dims[c];
        if (!on(b)) continue;
        int rc = axis(out, O, dims[b], I, cur, false, false);
        if (rc) return rc;
      }
      a = -1;
    }
    // the contiguous axis and its neighbour: two transposing passes when both
    // lengths have a specialised pass (every store is then a column tile)
    while (a >= 0 && !on(a)) --a;
    if (a >= 1 && tc_mode != 1) {
      int b = a - 1;
      while (b >= 0 && dims[b] == 1) --b;
      // only when the two axes are adjacent and transformed, and some outer
      // transformed axis remains to absorb the buffer parity (the pair itself
      // ends where it started)
      int outer = 0;
      for (int c = 0; c < b; ++c) outer += on(c);
      if (b >= 0 && !on(b)) b = -1;
      int64_t Ob = 1;
      for (int c = 0; c < b; ++c) Ob *= dims[c];
      if (b >= 0 && b == a - 1 && dims[b] == dims[a] && plane_cluster_step(out, Ob, dims[a], cur)) {
        a = b - 1;
      } else if (b >= 0 && b == a - 1 && outer > 0) {
        int64_t O = 1;
        for (int c = 0; c < b; ++c) O *= dims[c];
        if (dims[b] == dims[a] && plane_step(out, O, dims[a], cur))
          a = b - 1;
        else if (transposed_pair(out, O, dims[b], dims[a], cur, other_buf(cur), cur))
          a = b - 1;
      }
    }
    for (; a >= 0; --a) {
      int64_t I = 1, O = 1;
      for (int b = a + 1; b < ndim; ++b) I *= dims[b];
      for (int b = 0; b < a; ++b) O *= dims[b];
      if (!on(a)) continue;
      int rc = axis(out, O, dims[a], I, cur, false, false);
      if (rc) return rc;
    }
    if (out.empty()) {
      Step cp;
      cp.kind = ST_COPY;
      cp.in_buf = BUF_SRC;
      cp.out_buf = BUF_DST;
      int64_t t = 1;
      for (int b = 0; b < ndim; ++b) t *= dims[b];
      cp.total = t;
      out.push_back(cp);
      return 0;
    }
    if (out.back().out_buf == BUF_DST) return 0;
    // Parity fix: let the last in-place step (the first, with load_first)
    // write the other buffer instead, and exchange src/dst for every step
    // after it.
    const int nsteps = (int)out.size();
    for (int it = 0; it < nsteps; ++it) {
      const int i = load_first ? it : nsteps - 1 - it;
      Step& st = out[i];
      const bool user = (st.in_buf == BUF_SRC || st.in_buf == BUF_DST);
      const bool inplace_pass =
          (st.kind == ST_PASS || (st.kind == ST_PLANE && st.cluster)) && user && st.in_buf == st.out_buf;
      const bool demod = st.kind == ST_BS_DEMOD && (st.out_buf == BUF_SRC || st.out_buf == BUF_DST);
      if (inplace_pass || demod) {
        st.out_buf = other_buf(demod ? st.out_buf : st.in_buf);
        for (size_t j = i + 1; j < out.size(); ++j) {
          Step& t = out[j];
          if (t.in_buf == BUF_SRC || t.in_buf == BUF_DST) t.in_buf = other_buf(t.in_buf);
          if (t.out_buf == BUF_SRC || t.out_buf == BUF_DST) t.out_buf = other_buf(t.out_buf);
          if (t.kind == ST_PLANE) t.mid_buf = other_buf(t.mid_buf);
        }
        if (out.back().out_buf == BUF_DST) return 0;
        break;
      }
      // a Bluestein block writes its result to its input buffer through
      // scratch; the demodulate step above handles it
    }
    // last resort: copy
    Step cp;
    cp.kind = ST_COPY;
    cp.in_buf = out.back().out_buf;
    cp.out_buf = BUF_DST;
    int64_t t = 1;
    for (int b = 0; b < ndim; ++b) t *= dims[b];
    cp.total = t;
    out.push_back(cp);
    return 0;
  }
};

static void digit_tables(int L, std::vector<uint16_t>& p2k, std::vector<uint16_t>& k2p) {
  RadixPlan rp = radix_plan(L);
  p2k.assign(L, 0);
  k2p.assign(L, 0);
  for (int p = 0; p < L; ++p) {
    // p = sum_s d_s * m_s with m_s = L / (r_0 .. r_s); k = sum_s d_s * (r_0..r_{s-1})
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

}  // namespace shafft_sm100

using namespace shafft_sm100;

struct shafft_sm100_plan_s;
using Plan = shafft_sm100_plan_s;

struct shafft_sm100_plan_s {
  int precision = 0;
  int ndim = 0;
  std::vector<int64_t> dims;
  int64_t total = 0;
  std::vector<Step> steps;
  std::vector<LTable> ltabs;
  std::vector<NTable> ntabs;
  std::vector<BTable> btabs;
  size_t table_bytes = 0;
  unsigned char* d_tables = nullptr;
  int64_t scratch_elems = 0;
  void* d_s0 = nullptr;
  void* d_s1 = nullptr;
  cudaStream_t stream = nullptr;
  int device = 0;
  int flags = 0;
  size_t off_tcerr = 0;  // device error word of passes with bounded waits (0 = ok)
  bool check_err = false;  // some pass may set it (tensor-core or column passes)
  int map_fused = 0;       // exchange block maps fused: bit 0 load, bit 1 store
  // Replayed launch sequences: executes with the same (src, dst, direction,
  // scale) run as one CUDA graph from the third call on (the first runs
  // eagerly, the second is captured on a private stream).
  struct GraphEntry {
    void* src;
    void* dst;
    int dir;
    double scale;
    int calls;
    cudaGraphExec_t exec;
    uint64_t last;
  };
  std::vector<GraphEntry> graphs;
  cudaStream_t capture_stream = nullptr;
  bool graphs_off = false;
  uint64_t graph_clock = 0;
  int graph_evictions = 0;  // replay turns itself off for callers that cycle through many buffers
};

namespace {

template <typename T>
struct Launcher {
  using C = typename Vec2<T>::type;
  using K = Launch<T>;

  static int init_once() {
    const cudaError_t err = K::init_device();
    if (err != cudaSuccess) {
      g_last_cuda = (int)err;
      return set_err(SHAFFT_SM100_ECUDA, "kernel attribute setup: %s", cudaGetErrorString(err));
    }
    return 0;
  }

  static PassTables<C> tables(const shafft_sm100_plan_s* p, const Step& st) {
    PassTables<C> tb{};
    const LTable& lt = p->ltabs[st.tabL];
    tb.twL = reinterpret_cast<const C*>(p->d_tables + lt.off_tw);
    tb.p2k = reinterpret_cast<const uint16_t*>(p->d_tables + lt.off_p2k);
    tb.k2p = reinterpret_cast<const uint16_t*>(p->d_tables + lt.off_k2p);
    if (lt.tc_bytes) tb.tcB = p->d_tables + lt.off_tcB;
    if (st.g.bs_mode && st.tabB >= 0) {
      const BTable& bt = p->btabs[st.tabB];
      tb.bs_chirp = reinterpret_cast<const C*>(p->d_tables + bt.off_chirp);
      tb.bs_H = reinterpret_cast<const C*>(p->d_tables + bt.off_H);
    }
    if (st.tabN >= 0) {
      const NTable& nt = p->ntabs[st.tabN];
      tb.tw_hi = reinterpret_cast<const C*>(p->d_tables + nt.off_hi);
      tb.tw_lo = reinterpret_cast<const C*>(p->d_tables + nt.off_lo);
    }
    return tb;
  }

  static int check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
      g_last_cuda = (int)e;
      return set_err(SHAFFT_SM100_ECUDA, "%s launch: %s", what, cudaGetErrorString(e));
    }
    return 0;
  }

  static int pass(const shafft_sm100_plan_s* p, const Step& st, const void* in, void* out,
                  bool conj_in, bool conj_out, double scale, cudaStream_t s) {
    int rc = init_once();
    if (rc) return rc;
    PassGeom g = st.g;
    g.conj_in = conj_in;
    g.conj_out = conj_out;
    g.scale = scale;
    if (st.tabN >= 0) {
      const NTable& nt = p->ntabs[st.tabN];
      g.tw_shift = nt.shift;
      g.tw_mask = nt.mask;
    }
    if (st.tc) {
      if constexpr (std::is_same<T, float>::value) {
        int* err = reinterpret_cast<int*>(p->d_tables + p->off_tcerr);
        return tc_pass(g, reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), tables(p, st),
                       err, s);
      } else {
        return set_err(SHAFFT_SM100_ENOTSUP, "tensor-core pass on a complex128 plan");
      }
    }
    if (st.fast)
      return check(K::fast(g, st.fast_row != 0, reinterpret_cast<const C*>(in),
                           reinterpret_cast<C*>(out), tables(p, st),
                           reinterpret_cast<int*>(p->d_tables + p->off_tcerr), s),
                   "fast fft pass");
    return check(K::pass(g, reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), tables(p, st),
                         st.smem, s),
                 "fft pass");
  }

  static int plane_cluster(const shafft_sm100_plan_s* p, const Step& st, const void* in, void* out,
                           bool conj_in, bool conj_out, double scale, cudaStream_t s) {
    if constexpr (std::is_same<T, float>::value) {
      const LTable& lt = p->ltabs[st.tabL];
      const int64_t L = st.g.L;
      return check(plane_cluster_pass(reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), st.planes,
                                      L * L, L * L, reinterpret_cast<const C*>(p->d_tables + lt.off_tw),
                                      conj_in ? 1 : 0, conj_out ? 1 : 0, scale,
                                      reinterpret_cast<int*>(p->d_tables + p->off_tcerr), s),
                   "cluster plane pass");
    } else {
      return set_err(SHAFFT_SM100_ENOTSUP, "cluster plane pass on a complex128 plan");
    }
  }

  static int plane(const shafft_sm100_plan_s* p, const Step& st, const void* in, void* mid, void* out,
                   bool conj_in, bool conj_out, double scale, cudaStream_t s) {
    int rc = init_once();
    if (rc) return rc;
    PassGeom gx = st.g, gy = st.g2;
    gx.conj_in = conj_in;
    gx.conj_out = 0;
    gx.scale = 1.0;
    gy.conj_in = 0;
    gy.conj_out = conj_out;
    gy.scale = scale;
    int* ctl = reinterpret_cast<int*>(p->d_tables + st.off_ctl);
    return check(K::plane(gx, gy, reinterpret_cast<const C*>(in), reinterpret_cast<C*>(mid),
                          reinterpret_cast<C*>(out), tables(p, st), (int)st.planes, ctl, st.lag, s),
                 "plane pass");
  }

  static int elementwise(const shafft_sm100_plan_s* p, const Step& st, const void* in, void* out,
                         bool conj_in, bool conj_out, double scale, cudaStream_t s) {
    const C* cin = reinterpret_cast<const C*>(in);
    C* cout = reinterpret_cast<C*>(out);
    if (st.kind == ST_COPY)
      return check(K::scale_copy(cin, cout, st.total, (T)scale, (conj_in != conj_out) ? 1 : 0, s),
                   "copy");
    const BTable& bt = p->btabs[st.tabB];
    const C* chirp = reinterpret_cast<const C*>(p->d_tables + bt.off_chirp);
    const C* H = reinterpret_cast<const C*>(p->d_tables + bt.off_H);
    if (st.kind == ST_BS_MOD)
      return check(K::bs_modulate(cin, cout, st.bsL, st.bsM, st.bsI, st.total, chirp,
                                  conj_in ? 1 : 0, s),
                   "bluestein modulate");
    if (st.kind == ST_BS_MULH) return check(K::bs_mulh(cout, H, st.bsM, st.total, s), "bluestein multiply");
    return check(K::bs_demod(cin, cout, st.bsL, st.bsM, st.bsI, st.total, chirp, conj_out ? 1 : 0,
                             (T)scale, s),
                 "bluestein demodulate");
  }

  static int run_steps(const shafft_sm100_plan_s* p, const std::vector<Step>& steps, void* const bufs[4],
                       bool conj, double scale, cudaStream_t s, int only = -1) {
    const size_t n = steps.size();
    for (size_t i = 0; i < n; ++i) {
      if (only >= 0 && (size_t)only != i) continue;
      const Step& st = steps[i];
      const bool first = (i == 0), last = (i + 1 == n);
      const bool cin = first && conj;
      const bool cout = last && conj;
      const double sc = last ? scale : 1.0;
      int rc;
      // one NVTX range per launch (host-side markers for a profiler's
      // timeline; a no-op unless a tool is attached)
      nvtxRangePushA(step_label(st));
      if (st.kind == ST_PASS)
        rc = pass(p, st, bufs[st.in_buf], bufs[st.out_buf], cin, cout, sc, s);
      else if (st.kind == ST_PLANE && st.cluster)
        rc = plane_cluster(p, st, bufs[st.in_buf], bufs[st.out_buf], cin, cout, sc, s);
      else if (st.kind == ST_PLANE)
        rc = plane(p, st, bufs[st.in_buf], bufs[st.mid_buf], bufs[st.out_buf], cin, cout, sc, s);
      else
        rc = elementwise(p, st, bufs[st.in_buf], bufs[st.out_buf], cin, cout, sc, s);
      nvtxRangePop();
      if (rc) return rc;
    }
    return 0;
  }

  // Build every table of the plan on the device.
  // Every table of the plan, generated on the plan's stream with one
  // synchronisation at the end.  The digit tables are copied from pageable
  // host memory first, while the stream is still empty (such a copy waits
  // for the stream's earlier work before it starts; under a server's load
  // that wait is behind other transforms' kernels).
  static int build_tables(shafft_sm100_plan_s* p) {
    for (const LTable& lt : p->ltabs) {
      std::vector<uint16_t> p2k, k2p;
      digit_tables(lt.L, p2k, k2p);
      CUDA_TRY(cudaMemcpyAsync(p->d_tables + lt.off_p2k, p2k.data(), 2 * lt.L,
                               cudaMemcpyHostToDevice, p->stream));
      CUDA_TRY(cudaMemcpyAsync(p->d_tables + lt.off_k2p, k2p.data(), 2 * lt.L,
                               cudaMemcpyHostToDevice, p->stream));
    }
    for (const LTable& lt : p->ltabs) {
      if (lt.tc_bytes) {
        const int rc = tc_gen_table(p->d_tables + lt.off_tcB, lt.L, p->stream);
        if (rc) return rc;
      }
      int rc = check(K::gen_twiddle(reinterpret_cast<C*>(p->d_tables + lt.off_tw), lt.L, 1, lt.L,
                                    p->stream),
                     "twiddle generation");
      if (rc) return rc;
    }
    for (const NTable& nt : p->ntabs) {
      int rc = check(K::gen_twiddle(reinterpret_cast<C*>(p->d_tables + nt.off_hi), nt.nhi, nt.nlo,
                                    nt.N, p->stream),
                     "twiddle generation");
      if (rc) return rc;
      rc = check(K::gen_twiddle(reinterpret_cast<C*>(p->d_tables + nt.off_lo), nt.nlo, 1, nt.N,
                                p->stream),
                 "twiddle generation");
      if (rc) return rc;
    }
    for (const BTable& bt : p->btabs) {
      C* chirp = reinterpret_cast<C*>(p->d_tables + bt.off_chirp);
      int rc = check(K::gen_chirp(chirp, bt.L, p->stream), "chirp generation");
      if (rc) return rc;
      rc = check(K::gen_bs_kernel(reinterpret_cast<C*>(p->d_s0), chirp, bt.L, bt.M, p->stream),
                 "bluestein kernel generation");
      if (rc) return rc;
      void* bufs[4] = {nullptr, nullptr, p->d_s0, p->d_s1};
      rc = run_steps(p, bt.hsteps, bufs, false, 1.0 / (double)bt.M, p->stream);
      if (rc) return rc;
      CUDA_TRY(cudaMemcpyAsync(p->d_tables + bt.off_H, bufs[bt.hresult_buf], sizeof(C) * bt.M,
                               cudaMemcpyDeviceToDevice, p->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(p->stream));
    return 0;
  }
};

// L2 prefetch distance a pass step launches with (Launch<T>::fast_prefetch):
// plain specialised passes only
static int pass_prefetch(int precision, const Step& st) {
  if (!st.fast || st.tc || st.g.bs_mode || st.g.map_mode) return 0;
  return precision ? Launch<double>::fast_prefetch(st.g.L, st.g.in_row != 0)
                   : Launch<float>::fast_prefetch(st.g.L, st.g.in_row != 0);
}

std::string describe_steps(int precision, const std::vector<Step>& steps, int64_t total) {
  std::string s = "{\"precision\":" + std::to_string(precision) + ",\"elements\":" +
                  std::to_string(total) + ",\"steps\":[";
  for (size_t i = 0; i < steps.size(); ++i) {
    const Step& st = steps[i];
    char b[768];
    if (st.kind == ST_PLANE && st.cluster) {
      snprintf(b, sizeof(b),
               "{\"kind\":\"plane\",\"L\":%d,\"planes\":%lld,\"cluster\":16,\"in\":\"%s\",\"out\":\"%s\",\"smem\":%zu}",
               st.g.L, (long long)st.planes, buf_name(st.in_buf), buf_name(st.out_buf), st.smem);
    } else if (st.kind == ST_PLANE) {
      snprintf(b, sizeof(b),
               "{\"kind\":\"plane\",\"L\":%d,\"planes\":%lld,\"lag\":%d,\"in\":\"%s\",\"mid\":\"%s\",\"out\":\"%s\",\"fast\":1}",
               st.g.L, (long long)st.planes, st.lag, buf_name(st.in_buf), buf_name(st.mid_buf),
               buf_name(st.out_buf));
    } else if (st.kind == ST_PASS) {
      std::string rad;
      for (int r = 0; r < st.g.nst; ++r) rad += (r ? "," : "") + std::to_string(st.g.rad[r]);
      snprintf(b, sizeof(b),
               "{\"kind\":\"pass\",\"L\":%d,\"radices\":[%s],\"W\":%d,\"in\":\"%s\",\"out\":\"%s\","
               "\"in_row\":%d,\"out_row\":%d,\"tiles\":%lld,\"smem\":%zu,\"twiddle\":%d,"
               "\"ext\":[%lld,%lld,%lld,%lld],\"sn_in\":%lld,\"sk_out\":%lld,\"fast\":%d,\"tc\":%d,\"bs\":%d,"
               "\"map\":%d,\"prefetch\":%d}",
               st.g.L, rad.c_str(), st.g.W, buf_name(st.in_buf), buf_name(st.out_buf), st.g.in_row,
               st.g.out_row, (long long)st.g.ntiles, st.smem, st.g.tw_mode, (long long)st.g.ext[0],
               (long long)st.g.ext[1], (long long)st.g.ext[2], (long long)st.g.ext[3],
               (long long)st.g.sn_in, (long long)st.g.sk_out, st.fast, st.tc, st.g.bs_mode, st.g.map_mode,
               pass_prefetch(precision, st));
    } else {
      const char* k = st.kind == ST_BS_MOD    ? "bluestein_modulate"
                      : st.kind == ST_BS_MULH ? "bluestein_multiply"
                      : st.kind == ST_BS_DEMOD ? "bluestein_demodulate"
                                               : "copy";
      snprintf(b, sizeof(b), "{\"kind\":\"%s\",\"L\":%lld,\"M\":%lld,\"in\":\"%s\",\"out\":\"%s\",\"total\":%lld}",
               k, (long long)st.bsL, (long long)st.bsM, buf_name(st.in_buf), buf_name(st.out_buf),
               (long long)st.total);
    }
    if (i) s += ",";
    s += b;
  }
  s += "]}";
  return s;
}

int copy_out(const std::string& s, char* buf, int buflen) {
  if (!buf || buflen <= 0) return SHAFFT_SM100_EINVAL;
  if ((int)s.size() + 1 > buflen) {
    memcpy(buf, s.data(), buflen - 1);
    buf[buflen - 1] = 0;
    return set_err(SHAFFT_SM100_EINVAL, "description truncated (%zu bytes needed)", s.size() + 1);
  }
  memcpy(buf, s.c_str(), s.size() + 1);
  return 0;
}

// axes to transform as a bit mask; naxes < 0 or axes == NULL: every axis
int axes_mask(int ndim, int naxes, const int* axes, uint64_t* mask) {
  if (naxes < 0 || !axes) {
    *mask = ~0ull;
    return 0;
  }
  if (ndim > 64) return set_err(SHAFFT_SM100_ENOTSUP, "an axis subset needs ndim <= 64");
  uint64_t m = 0;
  for (int i = 0; i < naxes; ++i) {
    if (axes[i] < 0 || axes[i] >= ndim) return set_err(SHAFFT_SM100_EINVAL, "axis %d out of range", axes[i]);
    if ((m >> axes[i]) & 1ull) return set_err(SHAFFT_SM100_EINVAL, "axis %d listed twice", axes[i]);
    m |= 1ull << axes[i];
  }
  *mask = m;
  return 0;
}

// ---- plan creation with explicit planning choices ------------------------

struct Knobs {
  int balanced = -1;  // -1: by precision
  int widen = 1;
  int tc = -1;        // -1: as the flags say; 0: plain; 2: tensor cores on prime-factor axes
};

int effective_flags(int flags, const Knobs& k) {
  if (k.tc == 0) flags &= ~(SHAFFT_SM100_PLAN_TENSOR_CORE | SHAFFT_SM100_PLAN_TC_PRIME_AXES);
  if (k.tc == 2) flags = (flags & ~SHAFFT_SM100_PLAN_TENSOR_CORE) | SHAFFT_SM100_PLAN_TC_PRIME_AXES;
  return flags;
}

void configure(Planner& pl, const Knobs& k, uint64_t mask) {
  pl.axes_mask = mask;
  pl.balanced = k.balanced;
  pl.widen = k.widen;
}

// Exchange block maps asked for a plan's input and output
// (shafft_sm100_plan_create_axes_mapped): {outer, n, inner, parts} of the
// [outer][n][inner] array whose per-peer blocks the input is read from /
// the output is written to; parts = 0: none.
struct BlockMaps {
  int64_t load[4] = {0, 0, 0, 0};
  int64_t store[4] = {0, 0, 0, 0};
};

static bool map_valid(const int64_t m[4], int64_t total) {
  return m[0] >= 1 && m[2] >= 1 && m[3] >= 1 && m[1] >= m[3] && m[0] * m[1] * m[2] == total;
}

static int log2_exact(int64_t x) {
  if (x < 1 || (x & (x - 1))) return -1;
  int l = 0;
  while (((int64_t)1 << l) < x) ++l;
  return l;
}

// The fused form covers even partitions with power-of-two n, inner and
// parts (index arithmetic by shifts); others keep the separate kernels.
static bool map_fusable(const int64_t m[4]) {
  return log2_exact(m[1]) >= 0 && log2_exact(m[2]) >= 0 && log2_exact(m[3]) >= 0;
}

static void set_map(PassGeom& g, const int64_t m[4], int bit) {
  g.map_mode = bit;
  g.map_outer = m[0];
  g.map_log_n = log2_exact(m[1]);
  g.map_log_inner = log2_exact(m[2]);
  g.map_log_q = log2_exact(m[1] / m[3]);
}

// The loads or stores of a specialised pass take a block map when every
// access the kernel makes to that buffer stays inside one run that the map
// keeps contiguous: q * inner consecutive elements (q = n / parts, the
// block length), starting at a multiple of it.  The accesses are 16-byte
// chunks of vw elements for column tiles (offsets that are multiples of vw)
// and whole rows of L points for row tiles (offsets that are multiples of L).
static bool map_access_ok(const PassGeom& g, bool load, bool row_tile, int vw, int64_t run) {
  const int64_t unit = (load && row_tile) ? g.L : vw;
  if (run % unit) return false;
  const int64_t* st = load ? g.sin : g.sout;
  if (load && row_tile) {
    if (g.sn_in != 1) return false;
    for (int d = 0; d < 4; ++d)
      if (g.ext[d] > 1 && st[d] % unit) return false;
    return true;
  }
  if (st[0] != 1 || (load ? g.sn_in : g.sk_out) % unit) return false;
  for (int d = 1; d < 4; ++d)
    if (g.ext[d] > 1 && st[d] % unit) return false;
  return true;
}

// Fuse the requested maps into the first step's loads and the last step's
// stores where those are out-of-place specialised passes; returns the fused
// bits.  A step carries one map, so a one-step plan takes the store map.
static int apply_maps(std::vector<Step>& steps, const BlockMaps& m, int precision, int64_t total) {
  if (steps.empty()) return 0;
  const int vw = precision ? 1 : 2;
  int fused = 0;
  auto plain_fast = [](const Step& st) {
    return st.kind == ST_PASS && st.fast && !st.tc && st.g.bs_mode == 0 && st.g.map_mode == 0;
  };
  Step& last = steps.back();
  if (map_valid(m.store, total) && map_fusable(m.store) && plain_fast(last) && last.out_buf == BUF_DST &&
      last.in_buf != BUF_DST && map_access_ok(last.g, false, last.fast_row, vw, m.store[1] / m.store[3] * m.store[2])) {
    set_map(last.g, m.store, MAP_STORE);
    fused |= 2;
  }
  Step& first = steps.front();
  if (map_valid(m.load, total) && map_fusable(m.load) && plain_fast(first) && first.in_buf == BUF_SRC &&
      first.out_buf != BUF_SRC && map_access_ok(first.g, true, first.fast_row, vw, m.load[1] / m.load[3] * m.load[2])) {
    set_map(first.g, m.load, MAP_LOAD);
    fused |= 1;
  }
  return fused;
}

// The steps of a plan asked for block maps (planning only): the default
// planning, or the load_first one when it fuses more of the maps.
static int plan_with_maps(Planner& pl, std::vector<Step>& steps, int ndim, const int64_t* dims, int precision,
                          int flags, uint64_t mask, int64_t total, const Knobs& k, const BlockMaps& maps) {
  int rc = pl.plan_nd(steps, ndim, dims);
  if (rc || maps.load[3] == 0) return rc;
  Planner pl2(precision, flags);
  configure(pl2, k, mask);
  pl2.load_first = 1;
  std::vector<Step> steps2;
  if (pl2.plan_nd(steps2, ndim, dims) == 0) {
    std::vector<Step> t1 = steps, t2 = steps2;
    const int f1 = apply_maps(t1, maps, precision, total), f2 = apply_maps(t2, maps, precision, total);
    if (__builtin_popcount(f2) > __builtin_popcount(f1)) {
      pl = std::move(pl2);
      steps = std::move(steps2);
    }
  }
  return 0;
}

int create_plan(shafft_sm100_plan* out, int ndim, const int64_t* dims, int precision, int flags,
                uint64_t mask, int64_t total, const Knobs& k, const BlockMaps* maps = nullptr) {
  flags = effective_flags(flags, k);
  std::unique_ptr<shafft_sm100_plan_s> p(new (std::nothrow) shafft_sm100_plan_s());
  if (!p) return set_err(SHAFFT_SM100_EALLOC, "host allocation failed");
  p->precision = precision;
  p->ndim = ndim;
  p->dims.assign(dims, dims + ndim);
  p->total = total;
  p->flags = flags;
  Planner pl(precision, flags);
  configure(pl, k, mask);
  int rc = maps ? plan_with_maps(pl, p->steps, ndim, dims, precision, flags, mask, total, k, *maps)
                : pl.plan_nd(p->steps, ndim, dims);
  if (rc) return rc;
  bool cluster_steps = false;
  for (const Step& st : p->steps) cluster_steps |= (st.kind == ST_PLANE && st.cluster);
  if (cluster_steps && !plane_cluster_available()) {
    // this device cannot co-schedule the plane clusters: plan again without
    pl = Planner(precision, flags);
    configure(pl, k, mask);
    pl.plane_cluster_enabled = 0;
    rc = pl.plan_nd(p->steps, ndim, dims);
    if (rc) return rc;
  }
  if (maps) p->map_fused = apply_maps(p->steps, *maps, precision, total);
  p->off_tcerr = pl.off_tcerr;
  p->check_err = (flags & (SHAFFT_SM100_PLAN_TENSOR_CORE | SHAFFT_SM100_PLAN_TC_PRIME_AXES)) != 0;
  for (const Step& st : p->steps)
    if (st.kind == ST_PLANE && st.cluster) p->check_err = true;  // bounded prefetch waits
  // column passes can set it only through the opt-in bulk-copy kernel
  const char* tma = getenv("SHAFFT_SM100_TMA");
  if (tma && atoi(tma) != 0) {
    for (const Step& st : p->steps)
      if (st.fast && !st.fast_row) p->check_err = true;
    for (const BTable& bt : p->btabs)
      for (const Step& st : bt.hsteps)
        if (st.fast && !st.fast_row) p->check_err = true;
  }
  p->ltabs = pl.ltabs;
  p->ntabs = pl.ntabs;
  p->btabs = pl.btabs;
  p->table_bytes = std::max<size_t>(pl.table_bytes, 256);
  p->scratch_elems = pl.scratch_elems;
  CUDA_TRY(cudaGetDevice(&p->device));
  if (dev_malloc(reinterpret_cast<void**>(&p->d_tables), p->table_bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_err(SHAFFT_SM100_EALLOC, "cudaMalloc(%zu) for tables failed", p->table_bytes);
  }
  if (p->scratch_elems > 0) {
    const size_t b = (size_t)p->scratch_elems * (precision ? 16 : 8);
    if (dev_malloc(&p->d_s0, b) != cudaSuccess || dev_malloc(&p->d_s1, b) != cudaSuccess) {
      cudaGetLastError();
      dev_free(p->d_tables);
      if (p->d_s0) dev_free(p->d_s0);
      return set_err(SHAFFT_SM100_EALLOC, "cudaMalloc(%zu) for scratch failed", b);
    }
  }
  if (cudaMemset(p->d_tables, 0, p->table_bytes) != cudaSuccess) {
    cudaGetLastError();
    dev_free(p->d_tables);
    if (p->d_s0) dev_free(p->d_s0);
    if (p->d_s1) dev_free(p->d_s1);
    return set_err(SHAFFT_SM100_ECUDA, "cudaMemset of the plan tables failed");
  }
  rc = precision ? Launcher<double>::build_tables(p.get()) : Launcher<float>::build_tables(p.get());
  if (rc) {
    dev_free(p->d_tables);
    if (p->d_s0) dev_free(p->d_s0);
    if (p->d_s1) dev_free(p->d_s1);
    return rc;
  }
  *out = p.release();
  return 0;
}

// ---- measured planning (SHAFFT_SM100_PLAN_MEASURE) ------------------------
//
// The analogue of the reference's FFTW planner effort (SHAFFT_FFTW_PLANNER=
// MEASURE, src/cpp/fft/fftw_method/common/env.hpp:29-46): every distinct pass
// list the planning choices yield is built and timed (forward transforms of
// zeros on two scratch buffers, 2 warm-up + 5 timed, CUDA events), the
// fastest choice is kept and cached per shape in the text file
// SHAFFT_SM100_PLAN_CACHE (default ~/.cache/shafft_sm100_plans.txt).  The
// tensor-core alternative is only considered when the caller allowed it
// with SHAFFT_SM100_PLAN_TC_PRIME_AXES.  If the scratch buffers cannot be
// allocated the default choices are used.

std::mutex g_plan_cache_mu;

std::string plan_cache_path() {
  if (const char* e = getenv("SHAFFT_SM100_PLAN_CACHE")) return e;
  const char* home = getenv("HOME");
  return std::string(home ? home : ".") + "/.cache/shafft_sm100_plans.txt";
}

std::string plan_key(int ndim, const int64_t* dims, int precision, int flags, uint64_t mask) {
  std::string k = (precision ? "c128" : "c64") + std::string(":f") + std::to_string(flags) + ":m" +
                  std::to_string((unsigned long long)mask) + ":";
  for (int a = 0; a < ndim; ++a) k += (a ? "x" : "") + std::to_string((long long)dims[a]);
  return k;
}

bool cache_lookup(const std::string& key, Knobs* k) {
  std::lock_guard<std::mutex> lk(g_plan_cache_mu);
  FILE* f = fopen(plan_cache_path().c_str(), "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    char name[900];
    Knobs t;
    if (sscanf(line, "%899s %d %d %d", name, &t.balanced, &t.widen, &t.tc) == 4 && key == name) {
      *k = t;  // the last entry of a key wins
      found = true;
    }
  }
  fclose(f);
  return found;
}

void cache_store(const std::string& key, const Knobs& k) {
  std::lock_guard<std::mutex> lk(g_plan_cache_mu);
  const std::string path = plan_cache_path();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    const std::string dir = path.substr(0, slash);
    mkdir(dir.c_str(), 0755);  // best effort; an existing directory is fine
  }
  if (FILE* f = fopen(path.c_str(), "a")) {
    fprintf(f, "%s %d %d %d\n", key.c_str(), k.balanced, k.widen, k.tc);
    fclose(f);
  }
}

// forward time of a plan in ms (negative on failure)
double time_forward(shafft_sm100_plan p, void* a, void* b) {
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double ms = -1.0;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
      cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i) ok = shafft_sm100_execute(p, a, b, 0, 1.0, s) == 0;
    cudaEventRecord(e0, s);
    for (int i = 0; i < 5 && ok; ++i) ok = shafft_sm100_execute(p, a, b, 0, 1.0, s) == 0;
    cudaEventRecord(e1, s);
    float t = 0;
    if (ok && cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&t, e0, e1) == cudaSuccess &&
        shafft_sm100_plan_status(p) == 0)
      ms = t / 5.0;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaGetLastError();
  return ms;
}

Knobs measured_knobs(int ndim, const int64_t* dims, int precision, int flags, uint64_t mask,
                     int64_t total) {
  const std::string key = plan_key(ndim, dims, precision, flags, mask);
  Knobs best;
  if (cache_lookup(key, &best)) return best;
  std::vector<Knobs> cands;
  const bool tc_alt = precision == 0 && (flags & SHAFFT_SM100_PLAN_TC_PRIME_AXES) &&
                      !(flags & SHAFFT_SM100_PLAN_TENSOR_CORE);
  for (int bal : {1, 0})
    for (int wid : {1, 0})
      for (int tc : tc_alt ? std::vector<int>{0, 2} : std::vector<int>{-1}) {
        Knobs k;
        k.balanced = bal;
        k.widen = wid;
        k.tc = tc;
        cands.push_back(k);
      }
  // keep one candidate per distinct pass list
  std::vector<Knobs> distinct;
  std::vector<std::string> seen;
  for (const Knobs& k : cands) {
    Planner pl(precision, effective_flags(flags, k));
    configure(pl, k, mask);
    std::vector<Step> steps;
    if (pl.plan_nd(steps, ndim, dims)) continue;
    const std::string d = describe_steps(precision, steps, total);
    if (std::find(seen.begin(), seen.end(), d) != seen.end()) continue;
    seen.push_back(d);
    distinct.push_back(k);
  }
  if (distinct.size() <= 1) return distinct.empty() ? Knobs{} : distinct[0];
  const size_t bytes = (size_t)total * (precision ? 16 : 8);
  void *a = nullptr, *b = nullptr;
  if (cudaMalloc(&a, bytes) != cudaSuccess || cudaMalloc(&b, bytes) != cudaSuccess) {
    cudaGetLastError();
    if (a) cudaFree(a);
    return Knobs{};
  }
  cudaMemset(a, 0, bytes);
  double best_ms = -1.0;
  best = distinct[0];
  for (const Knobs& k : distinct) {
    shafft_sm100_plan p = nullptr;
    if (create_plan(&p, ndim, dims, precision, flags, mask, total, k)) continue;
    const double ms = time_forward(p, a, b);
    shafft_sm100_plan_destroy(p);
    if (ms >= 0 && (best_ms < 0 || ms < best_ms)) {
      best_ms = ms;
      best = k;
    }
  }
  cudaFree(a);
  cudaFree(b);
  if (best_ms >= 0) cache_store(key, best);
  return best;
}

// SHAFFT_SM100_GRAPHS=0 turns graph replay of executes off
bool graphs_enabled() {
  static const bool on = [] {
    const char* e = getenv("SHAFFT_SM100_GRAPHS");
    return !(e && atoi(e) == 0);
  }();
  return on;
}

int validate_flags(int flags, int precision) {
  const int tc_flags = SHAFFT_SM100_PLAN_TENSOR_CORE | SHAFFT_SM100_PLAN_TC_PRIME_AXES;
  if (flags & ~(tc_flags | SHAFFT_SM100_PLAN_MEASURE))
    return set_err(SHAFFT_SM100_EINVAL, "unknown plan flags");
  if ((flags & tc_flags) && precision != 0)
    return set_err(SHAFFT_SM100_ENOTSUP, "the tensor-core form is complex64 only");
  return 0;
}

int validate_dims(int ndim, const int64_t* dims, int precision, int64_t* total) {
  if (ndim < 1 || ndim > 64 || !dims) return set_err(SHAFFT_SM100_EINVAL, "bad ndim/dims");
  if (precision != 0 && precision != 1) return set_err(SHAFFT_SM100_EINVAL, "bad precision");
  int64_t t = 1;
  for (int a = 0; a < ndim; ++a) {
    if (dims[a] < 1) return set_err(SHAFFT_SM100_EINVAL, "dims[%d] = %lld < 1", a, (long long)dims[a]);
    if (t > (int64_t(1) << 42) / dims[a]) return set_err(SHAFFT_SM100_ENOTSUP, "tensor too large");
    t *= dims[a];
  }
  *total = t;
  return 0;
}

}  // namespace

// The passes move 16-byte vectors (two complex64 or one complex128 element)
// and bulk tensor copies need 16-byte aligned sources: a buffer that is not
// would fault the context, so the entry points refuse it.
static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
static int misaligned() {
  return set_err(SHAFFT_SM100_EINVAL,
                 "src and dst must be 16-byte aligned (cudaMalloc and shafftAllocBuffer memory is)");
}

namespace shafft_sm100 {
static std::atomic<int64_t> g_tma_launches{0};
void count_tma_launch() { g_tma_launches.fetch_add(1, std::memory_order_relaxed); }

bool plan_shareable(const shafft_sm100_plan_s* plan) {
  if (!plan || plan->scratch_elems > 0) return false;
  for (const Step& st : plan->steps)
    if (st.kind == ST_PLANE) return false;  // zeroes and counts its control words every launch
  return true;
}
}  // namespace shafft_sm100

extern "C" {

int shafft_sm100_plan_query(int ndim, const int64_t* dims, int precision, char* buf, int buflen) {
  return shafft_sm100_plan_query_ex(ndim, dims, precision, 0, buf, buflen);
}

int shafft_sm100_plan_query_ex(int ndim, const int64_t* dims, int precision, int flags, char* buf,
                               int buflen) {
  return shafft_sm100_plan_query_axes(ndim, dims, precision, flags, -1, nullptr, buf, buflen);
}

int shafft_sm100_plan_query_axes(int ndim, const int64_t* dims, int precision, int flags, int naxes,
                                 const int* axes, char* buf, int buflen) {
  int64_t total = 0;
  int rc = validate_flags(flags, precision);
  if (rc) return rc;
  rc = validate_dims(ndim, dims, precision, &total);
  if (rc) return rc;
  uint64_t mask = 0;
  rc = axes_mask(ndim, naxes, axes, &mask);
  if (rc) return rc;
  // a measured plan is described with its cached choice (no measuring here)
  const char* env = getenv("SHAFFT_SM100_PLANNER");
  const bool measure = (flags & SHAFFT_SM100_PLAN_MEASURE) || (env && strcmp(env, "MEASURE") == 0);
  flags &= ~SHAFFT_SM100_PLAN_MEASURE;
  Knobs k;
  if (measure) cache_lookup(plan_key(ndim, dims, precision, flags, mask), &k);
  flags = effective_flags(flags, k);
  Planner pl(precision, flags);
  configure(pl, k, mask);
  std::vector<Step> steps;
  rc = pl.plan_nd(steps, ndim, dims);
  if (rc) return rc;
  return copy_out(describe_steps(precision, steps, total), buf, buflen);
}

int shafft_sm100_plan_create_nd(shafft_sm100_plan* out, int ndim, const int64_t* dims, int precision) {
  return shafft_sm100_plan_create_nd_ex(out, ndim, dims, precision, 0);
}

int shafft_sm100_plan_create_nd_ex(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                   int precision, int flags) {
  return shafft_sm100_plan_create_axes(out, ndim, dims, precision, flags, -1, nullptr);
}

int shafft_sm100_plan_create_axes(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                  int precision, int flags, int naxes, const int* axes) {
  if (!out) return set_err(SHAFFT_SM100_EINVAL, "null plan pointer");
  *out = nullptr;
  int64_t total = 0;
  int rc = validate_flags(flags, precision);
  if (rc) return rc;
  rc = validate_dims(ndim, dims, precision, &total);
  if (rc) return rc;
  uint64_t mask = 0;
  rc = axes_mask(ndim, naxes, axes, &mask);
  if (rc) return rc;
  const char* env = getenv("SHAFFT_SM100_PLANNER");
  const bool measure = (flags & SHAFFT_SM100_PLAN_MEASURE) || (env && strcmp(env, "MEASURE") == 0);
  flags &= ~SHAFFT_SM100_PLAN_MEASURE;
  Knobs k;
  if (measure) k = measured_knobs(ndim, dims, precision, flags, mask, total);
  return create_plan(out, ndim, dims, precision, flags, mask, total, k);
}

int shafft_sm100_plan_create_axes_mapped(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                         int precision, int flags, int naxes, const int* axes,
                                         const int64_t* load_map, const int64_t* store_map, int* fused) {
  if (!out) return set_err(SHAFFT_SM100_EINVAL, "null plan pointer");
  *out = nullptr;
  if (fused) *fused = 0;
  int64_t total = 0;
  int rc = validate_flags(flags, precision);
  if (rc) return rc;
  rc = validate_dims(ndim, dims, precision, &total);
  if (rc) return rc;
  uint64_t mask = 0;
  rc = axes_mask(ndim, naxes, axes, &mask);
  if (rc) return rc;
  BlockMaps m;
  for (int i = 0; i < 4; ++i) {
    if (load_map) m.load[i] = load_map[i];
    if (store_map) m.store[i] = store_map[i];
  }
  for (const int64_t* q : {m.load, m.store})
    if (q[3] != 0 && !map_valid(q, total))
      return set_err(SHAFFT_SM100_EINVAL, "block map {%lld, %lld, %lld, %lld} does not cover the %lld elements",
                     (long long)q[0], (long long)q[1], (long long)q[2], (long long)q[3], (long long)total);
  flags &= ~SHAFFT_SM100_PLAN_MEASURE;
  rc = create_plan(out, ndim, dims, precision, flags, mask, total, Knobs{}, &m);
  if (!rc && fused) *fused = (*out)->map_fused;
  return rc;
}

int shafft_sm100_plan_query_mapped(int ndim, const int64_t* dims, int precision, int naxes, const int* axes,
                                   const int64_t* load_map, const int64_t* store_map, char* buf, int buflen) {
  int64_t total = 0;
  int rc = validate_dims(ndim, dims, precision, &total);
  if (rc) return rc;
  uint64_t mask = 0;
  rc = axes_mask(ndim, naxes, axes, &mask);
  if (rc) return rc;
  BlockMaps m;
  for (int i = 0; i < 4; ++i) {
    if (load_map) m.load[i] = load_map[i];
    if (store_map) m.store[i] = store_map[i];
  }
  for (const int64_t* q : {m.load, m.store})
    if (q[3] != 0 && !map_valid(q, total)) return set_err(SHAFFT_SM100_EINVAL, "block map does not cover the tensor");
  Planner pl(precision, 0);
  configure(pl, Knobs{}, mask);
  std::vector<Step> steps;
  rc = plan_with_maps(pl, steps, ndim, dims, precision, 0, mask, total, Knobs{}, m);
  if (rc) return rc;
  const int fused = apply_maps(steps, m, precision, total);
  std::string d = describe_steps(precision, steps, total);
  d.pop_back();  // the closing brace
  d += ",\"fused\":" + std::to_string(fused) + "}";
  return copy_out(d, buf, buflen);
}

int shafft_sm100_plan_create_1d(shafft_sm100_plan* out, int64_t n, int precision) {
  return shafft_sm100_plan_create_nd(out, 1, &n, precision);
}

int shafft_sm100_plan_destroy(shafft_sm100_plan plan) {
  if (!plan) return 0;
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != plan->device) cudaSetDevice(plan->device);
  for (auto& g : plan->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (plan->capture_stream) cudaStreamDestroy(plan->capture_stream);
  int rc = 0;
  for (void* q : {static_cast<void*>(plan->d_tables), plan->d_s0, plan->d_s1}) {
    const int r = q ? dev_free(q) : 0;  // reports changed guard bytes under SHAFFT_SM100_CANARY
    if (!rc) rc = r;
  }
  if (dev >= 0 && dev != plan->device) cudaSetDevice(dev);
  delete plan;
  return rc;
}

int shafft_sm100_set_stream(shafft_sm100_plan plan, void* stream) {
  if (!plan) return set_err(SHAFFT_SM100_EINVAL, "null plan");
  plan->stream = reinterpret_cast<cudaStream_t>(stream);
  return 0;
}

int shafft_sm100_execute(shafft_sm100_plan plan, void* src, void* dst, int direction, double scale,
                         void* stream) {
  if (!plan) return set_err(SHAFFT_SM100_EINVAL, "null plan");
  if (!src || !dst) return set_err(SHAFFT_SM100_EINVAL, "null buffer");
  if (src == dst) return set_err(SHAFFT_SM100_EINVAL, "src and dst must be distinct buffers");
  if (!aligned16(src) || !aligned16(dst)) return misaligned();
  if (direction != 0 && direction != 1) return set_err(SHAFFT_SM100_EINVAL, "bad direction");
  cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : plan->stream;
  void* bufs[4] = {src, dst, plan->d_s0, plan->d_s1};
  auto eager = [&](cudaStream_t st) {
    return plan->precision
               ? Launcher<double>::run_steps(plan, plan->steps, bufs, direction == 1, scale, st)
               : Launcher<float>::run_steps(plan, plan->steps, bufs, direction == 1, scale, st);
  };
  if (!graphs_enabled() || plan->graphs_off || plan->steps.size() < 2) return eager(s);
  // a caller that is itself capturing a graph gets plain launches
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return eager(s);
  }
  Plan::GraphEntry* e = nullptr;
  for (auto& g : plan->graphs)
    if (g.src == src && g.dst == dst && g.dir == direction && g.scale == scale) e = &g;
  if (!e) {
    if (plan->graphs.size() >= 8 && ++plan->graph_evictions > 8) {
      // the caller cycles through more (src, dst) pairs than the plan keeps:
      // captures would rarely be replayed, so run eagerly from now on
      for (auto& g : plan->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
      plan->graphs.clear();
      plan->graphs_off = true;
      return eager(s);
    }
    if (plan->graphs.size() >= 8) {  // evict the least recently used
      auto lru = std::min_element(plan->graphs.begin(), plan->graphs.end(),
                                  [](const Plan::GraphEntry& x, const Plan::GraphEntry& y) { return x.last < y.last; });
      if (lru->exec) cudaGraphExecDestroy(lru->exec);
      plan->graphs.erase(lru);
    }
    plan->graphs.push_back(Plan::GraphEntry{src, dst, direction, scale, 0, nullptr, 0});
    e = &plan->graphs.back();
  }
  e->last = ++plan->graph_clock;
  if (e->exec) {
    const cudaError_t r = cudaGraphLaunch(e->exec, s);
    if (r == cudaSuccess) return 0;
    cudaGetLastError();
    plan->graphs_off = true;
    return eager(s);
  }
  if (++e->calls < 2) return eager(s);
  // second call: capture the launch sequence once, then replay it on s
  if (!plan->capture_stream &&
      cudaStreamCreateWithFlags(&plan->capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    plan->graphs_off = true;
    return eager(s);
  }
  cudaGraph_t graph = nullptr;
  int rc = 0;
  bool ok = cudaStreamBeginCapture(plan->capture_stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    rc = eager(plan->capture_stream);
    ok = cudaStreamEndCapture(plan->capture_stream, &graph) == cudaSuccess && rc == 0 && graph;
  }
  if (ok) ok = cudaGraphInstantiate(&e->exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    cudaGetLastError();
    e->exec = nullptr;
    plan->graphs_off = true;
    return eager(s);
  }
  if (cudaGraphLaunch(e->exec, s) != cudaSuccess) {
    cudaGetLastError();
    plan->graphs_off = true;
    return eager(s);
  }
  return 0;
}

int shafft_sm100_execute_step(shafft_sm100_plan plan, int step, void* src, void* dst, int direction,
                              double scale, void* stream) {
  if (!plan) return set_err(SHAFFT_SM100_EINVAL, "null plan");
  if (step < 0 || step >= (int)plan->steps.size()) return set_err(SHAFFT_SM100_EINVAL, "bad step");
  if (!src || !dst || src == dst) return set_err(SHAFFT_SM100_EINVAL, "bad buffers");
  if (!aligned16(src) || !aligned16(dst)) return misaligned();
  cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : plan->stream;
  void* bufs[4] = {src, dst, plan->d_s0, plan->d_s1};
  return plan->precision
             ? Launcher<double>::run_steps(plan, plan->steps, bufs, direction == 1, scale, s, step)
             : Launcher<float>::run_steps(plan, plan->steps, bufs, direction == 1, scale, s, step);
}

int64_t shafft_sm100_step_bytes(shafft_sm100_plan plan, int step) {
  if (!plan || step < 0 || step >= (int)plan->steps.size()) return 0;
  const Step& st = plan->steps[step];
  const int64_t es = plan->precision ? 16 : 8;
  if (st.kind == ST_PLANE) return 2 * st.planes * st.g.L * st.g.L * es;
  if (st.kind == ST_PASS) {
    int64_t n = (int64_t)st.g.L;
    for (int d = 0; d < 4; ++d) n *= st.g.ext[d];
    if (st.g.bs_mode & (BS_LOAD_MOD | BS_STORE_DEMOD)) {
      // the x side of a fused modulate / demodulate touches bs_L of every
      // 2^bs_logM points
      const int64_t xb = (n >> st.g.bs_logM) * st.g.bs_L;
      const int64_t rd = (st.g.bs_mode & BS_LOAD_MOD) ? xb : n;
      const int64_t wr = (st.g.bs_mode & BS_STORE_DEMOD) ? xb : n;
      return (rd + wr) * es;
    }
    return 2 * n * es;
  }
  if (st.kind == ST_BS_MOD) return (st.total / st.bsM * st.bsL + st.total) * es;
  if (st.kind == ST_BS_DEMOD) return (st.total / st.bsL * st.bsL + st.total) * es;
  return 2 * st.total * es;
}

int shafft_sm100_scale(void* data, size_t count, int precision, double factor, void* stream) {
  if (!data && count) return set_err(SHAFFT_SM100_EINVAL, "null buffer");
  if (precision != 0 && precision != 1) return set_err(SHAFFT_SM100_EINVAL, "bad precision");
  if (count == 0) return 0;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = (int64_t)count;
  cudaError_t e;
  if (precision)
    e = Launch<double>::scale_copy(reinterpret_cast<const double2*>(data),
                                   reinterpret_cast<double2*>(data), n, factor, 0, s);
  else
    e = Launch<float>::scale_copy(reinterpret_cast<const float2*>(data),
                                  reinterpret_cast<float2*>(data), n, (float)factor, 0, s);
  CUDA_TRY(e);
  return 0;
}

int64_t shafft_sm100_tma_launch_count(void) { return shafft_sm100::g_tma_launches.load(); }

int shafft_sm100_plan_status(shafft_sm100_plan plan) {
  if (!plan) return set_err(SHAFFT_SM100_EINVAL, "null plan");
  if (plan->check_err) {
    int flag = 0;
    CUDA_TRY(cudaMemcpy(&flag, plan->d_tables + plan->off_tcerr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag)
      return set_err(SHAFFT_SM100_ECUDA,
                     "a pass gave up waiting (tensor-core MMA results or a bulk copy)");
  }
  for (const Step& st : plan->steps) {
    if (st.kind != ST_PLANE || st.cluster) continue;
    int flag = 0;
    CUDA_TRY(cudaMemcpy(&flag, plan->d_tables + st.off_ctl + 2 * sizeof(int), sizeof(int),
                        cudaMemcpyDeviceToHost));
    if (flag)
      return set_err(SHAFFT_SM100_ECUDA,
                     "fused plane pass: a wait for a plane's first-axis tiles timed out");
  }
  return 0;
}

int64_t shafft_sm100_plan_elements(shafft_sm100_plan plan) { return plan ? plan->total : 0; }

int shafft_sm100_plan_passes(shafft_sm100_plan plan) {
  if (!plan) return 0;
  int n = 0;
  for (const Step& st : plan->steps) n += (st.kind == ST_COPY) ? 1 : 1;
  return n;
}

int shafft_sm100_plan_launches(shafft_sm100_plan plan) { return plan ? (int)plan->steps.size() : 0; }

size_t shafft_sm100_plan_device_bytes(shafft_sm100_plan plan) {
  if (!plan) return 0;
  return plan->table_bytes + 2 * (size_t)plan->scratch_elems * (plan->precision ? 16 : 8);
}

int shafft_sm100_plan_describe(shafft_sm100_plan plan, char* buf, int buflen) {
  if (!plan) return set_err(SHAFFT_SM100_EINVAL, "null plan");
  return copy_out(describe_steps(plan->precision, plan->steps, plan->total), buf, buflen);
}

int shafft_sm100_malloc(void** ptr, size_t bytes) {
  if (!ptr) return set_err(SHAFFT_SM100_EINVAL, "null pointer");
  *ptr = nullptr;
  cudaError_t e = dev_malloc(ptr, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    g_last_cuda = (int)e;
    *ptr = nullptr;
    return set_err(SHAFFT_SM100_EALLOC, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return 0;
}

int shafft_sm100_free(void* ptr) {
  if (!ptr) return 0;
  return dev_free(ptr);
}

int shafft_sm100_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream) {
  if (!bytes) return 0;
  if (!dst || !src) return set_err(SHAFFT_SM100_EINVAL, "null pointer");
  cudaMemcpyKind k = kind == SHAFFT_SM100_H2D   ? cudaMemcpyHostToDevice
                     : kind == SHAFFT_SM100_D2H ? cudaMemcpyDeviceToHost
                     : kind == SHAFFT_SM100_D2D ? cudaMemcpyDeviceToDevice
                                                : cudaMemcpyDefault;
  if (stream) {
    CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, k, reinterpret_cast<cudaStream_t>(stream)));
  } else {
    CUDA_TRY(cudaMemcpy(dst, src, bytes, k));
  }
  return 0;
}

int shafft_sm100_stream_sync(void* stream) {
  CUDA_TRY(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)));
  return 0;
}

int shafft_sm100_device_name(char* buf, int buflen) {
  if (!buf || buflen <= 0) return set_err(SHAFFT_SM100_EINVAL, "bad buffer");
  buf[0] = 0;
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
  snprintf(buf, buflen, "%s", prop.name);
  return 0;
}

int shafft_sm100_last_cuda_error(void) { return g_last_cuda; }

const char* shafft_sm100_last_error_message(void) { return g_last_msg; }

const char* shafft_sm100_version(void) { return "shafft-sm100 0.1.0 (sm_100a)"; }

}  // extern "C"
