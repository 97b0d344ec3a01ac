// Specialised HBM pass for hot lengths (compile-time L and radix plan).
//
// One CTA transforms a tile of L points x W batch columns, W = 8 * VW where a
// 16-byte "chunk" holds VW complex elements (VW = 2 for complex64, 1 for
// complex128), so a tile row is exactly one 128-byte line.
//
// Phase A  every thread issues all the loads of its first-stage butterflies
//          before any arithmetic (R0 * NB0 * VW independent loads in flight
//          per thread), runs the radix-R0 butterflies in registers, applies
//          the DIF twiddle and stores 16-byte chunks to shared memory.
//          IN_ROW = false: the batch column is contiguous in HBM (column
//          tile) -- 8 lanes read one 128-byte line per instruction.
//          IN_ROW = true : the transform axis is contiguous (row tile) -- 32
//          lanes read 32 consecutive points of one row per instruction.
// Phase B  middle radix stages in shared memory.
// Phase C  last radix stage; the result is written straight from registers
//          to HBM in natural (digit-unreversed) order, 8 lanes per 128-byte
//          line, with scale / conjugation / four-step post-twiddle fused.
//          The output is always a column tile, so with IN_ROW the pass also
//          transposes (rotate-on-write).
// Shared layout: row p holds 8 chunks; chunk c of row p is stored at slot
// c ^ (p & 7).  Any 8 lanes that touch 8 different chunks of one row, or the
// same chunk of 8 rows with distinct p mod 8, hit 8 different 16-byte bank
// groups, so every phase is free of bank conflicts.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "butterflies.cuh"
#include "pass.h"

namespace shafft_sm100 {

template <typename T>
struct ChunkT;
template <>
struct ChunkT<float> {
  static constexpr int VW = 2;
};
template <>
struct ChunkT<double> {
  static constexpr int VW = 1;
};

template <int L, int R0, int R1, int R2, int NT>
struct FastCfg {
  static constexpr int S = (R2 > 1) ? 3 : 2;
  static_assert(R0 * R1 * (R2 > 1 ? R2 : 1) == L, "radices must multiply to L");
  static constexpr int NB0 = L * 8 / (R0 * NT);
  static constexpr int NB1 = L * 8 / (R1 * NT);
  static constexpr int NB2 = (R2 > 1) ? L * 8 / (R2 * NT) : 1;
  static_assert(NB0 >= 1 && NB0 * R0 * NT == L * 8, "stage 0 must tile the threads");
  static_assert(NB1 >= 1 && NB1 * R1 * NT == L * 8, "stage 1 must tile the threads");
  static_assert(R2 <= 1 || (NB2 >= 1 && NB2 * R2 * NT == L * 8), "stage 2 must tile the threads");
};

// 16-byte chunk I/O
template <typename C, int VW>
struct Chunk {
  C v[VW];
};

__device__ __forceinline__ int swz(int p, int c) { return p * 8 + (c ^ (p & 7)); }
// Layout of a tile whose phase A reads it from shared memory (a bulk tensor
// copy put it there as dense 128-byte rows): no XOR swizzle.  In a column
// tile every phase has 8 lanes on the 8 chunks of one row, so it is free of
// bank conflicts too.
template <bool SW>
__device__ __forceinline__ int sidx(int p, int c) {
  return SW ? swz(p, c) : p * 8 + c;
}

// Streaming (evict-first) global accesses for the tensor, so that the small
// twiddle table stays resident in L1; twiddles use the read-only path.
template <typename C>
__device__ __forceinline__ C ld_stream(const C* p);
template <>
__device__ __forceinline__ float2 ld_stream<float2>(const float2* p) { return __ldcs(p); }
template <>
__device__ __forceinline__ double2 ld_stream<double2>(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_chunk(const void* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
// The same load asking L2 to fetch the whole 256-byte block around the line
// (the neighbouring column tile's line comes with it).
__device__ __forceinline__ float4 ld_chunk_256(const void* p) {
  float4 v;
  asm volatile("ld.global.cs.L2::256B.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}
__device__ __forceinline__ void st_chunk(void* p, float4 v) { __stcs(reinterpret_cast<float4*>(p), v); }
template <typename C>
__device__ __forceinline__ C ld_tw(const C* p) { return __ldg(p); }

// Cache policy of a tile's HBM traffic.
//   LD_STREAM : input read once from HBM, evict-first in L1/L2
//   LD_L2     : input produced moments ago by another CTA; read at L2 only
enum TileLoad : int { LD_STREAM = 0, LD_L2 = 1 };
//   ST_STREAM : final output, evict-first
//   ST_KEEP   : intermediate that another CTA reads next; default policy
enum TileStore : int { ST_STREAM = 0, ST_KEEP = 1 };
// LDP/STP = POLICY_RUNTIME: policies (and the L2 discard) come from the
// runtime `pol` argument of fast_tile, so one instantiation serves several
// tile kinds.
constexpr int POLICY_RUNTIME = 2;
struct TilePolicy {
  int ld, st, discard;
};

template <typename C>
__device__ __forceinline__ C ld_l2(const C* p);
template <>
__device__ __forceinline__ float2 ld_l2<float2>(const float2* p) { return __ldcg(p); }
template <>
__device__ __forceinline__ double2 ld_l2<double2>(const double2* p) { return __ldcg(p); }

// Drop a 128-byte line from L2 without writing it back (its contents were
// consumed and will be overwritten before they are read again).
__device__ __forceinline__ void discard_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// Base offsets of tile `tile` of a specialised pass (W = 8 * VW columns).
struct FastTileAt {
  int64_t w0, bin, bout, tconst;
};
template <int W>
__device__ __forceinline__ FastTileAt fast_tile_at(const PassGeom& g, int64_t tile) {
  const int64_t tw = tile % g.tiles_w;
  int64_t rest = tile / g.tiles_w;
  const int64_t i1 = rest % g.ext[1];
  rest /= g.ext[1];
  const int64_t i2 = rest % g.ext[2];
  const int64_t i3 = rest / g.ext[2];
  FastTileAt a;
  a.w0 = tw * W;
  a.bin = a.w0 * g.sin[0] + i1 * g.sin[1] + i2 * g.sin[2] + i3 * g.sin[3];
  a.bout = a.w0 + i1 * g.sout[1] + i2 * g.sout[2] + i3 * g.sout[3];
  a.tconst = g.tw_dim == 1 ? i1 : (g.tw_dim == 2 ? i2 : (g.tw_dim == 3 ? i3 : 0));
  return a;
}

// Phase-A inputs of one tile: the R0 points of each of this thread's first-
// stage butterflies, held in registers from the loads to the first stage.
template <typename T, int L, int R0, int R1, int R2, int NT>
struct FastRegs {
  typename Cx<T>::type v[FastCfg<L, R0, R1, R2, NT>::NB0][R0][ChunkT<T>::VW];
};

// chunk-butterfly b of this thread: first-stage butterfly j, chunk column c
template <int L, int R0, int NT, bool IN_ROW>
__device__ __forceinline__ void fast_butterfly(int b, int& j, int& c) {
  constexpr int M0 = L / R0;
  const int id = threadIdx.x + b * NT;  // chunk-butterfly id in [0, M0*8)
  if (IN_ROW) {
    j = id % M0;
    c = id / M0;
  } else {
    c = id & 7;
    j = id >> 3;
  }
}

// Block-layout index of natural index v (PassGeom::map_*, pass.h).
__device__ __forceinline__ int64_t map_block(const PassGeom& g, int64_t v) {
  const int64_t i = v & (((int64_t)1 << g.map_log_inner) - 1);
  const int64_t t = v >> g.map_log_inner;
  const int64_t k = t & (((int64_t)1 << g.map_log_n) - 1);
  const int64_t o = t >> g.map_log_n;
  const int64_t p = k >> g.map_log_q, kk = k & (((int64_t)1 << g.map_log_q) - 1);
  return ((((p * g.map_outer + o) << g.map_log_q) + kk) << g.map_log_inner) + i;
}

// Extended instantiations of the specialised pass (template argument EXT).
enum FastExtKind : int { EXT_BS = 1, EXT_MAP = 2 };

// Phase A loads: issue every input load of tile `tile` into R (column
// tiles with FETCH = 256: 256-byte L2 fetches).
// EXT instantiations only: column tiles with PassGeom::bs_mode & BS_LOAD_MOD
// read the Bluestein modulation of x on the fly (see pass.h; `chirp` is its
// table), and map_mode & MAP_LOAD reads the input from an exchange's block
// layout.  The plain instantiations carry none of this code: a runtime test
// of bs_mode alone slowed the 512-point pass by a quarter; the two kinds are
// separate instantiations so that each keeps its own register budget.
template <typename T, int L, int R0, int R1, int R2, int NT, bool IN_ROW, bool SMEM_A = false, int EXT = 0,
          int FETCH = 0>
__device__ __forceinline__ void fast_load(const PassGeom& g, const typename Cx<T>::type* in, int64_t tile,
                                          const float4* sm, int LDP, FastRegs<T, L, R0, R1, R2, NT>& R,
                                          const typename Cx<T>::type* chirp = nullptr) {
  using C = typename Cx<T>::type;
  using Cfg = FastCfg<L, R0, R1, R2, NT>;
  constexpr int VW = ChunkT<T>::VW;
  constexpr int W = 8 * VW;
  const int64_t bin = fast_tile_at<W>(g, tile).bin;
  constexpr int M0 = L / R0;  // stride between the inputs of one butterfly
  int bj[Cfg::NB0], bc[Cfg::NB0];
#pragma unroll
  for (int b = 0; b < Cfg::NB0; ++b) fast_butterfly<L, R0, NT, IN_ROW>(b, bj[b], bc[b]);
  // issue every load first
#pragma unroll
  for (int b = 0; b < Cfg::NB0; ++b) {
#pragma unroll
    for (int r = 0; r < R0; ++r) {
      const int n = bj[b] + r * M0;
      if (IN_ROW) {
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          int64_t row = bin + (int64_t)(bc[b] * VW + e) * g.sin[0];
          // a row of L points lies in one contiguous run of the map (the planner checks)
          if ((EXT & EXT_MAP) && (g.map_mode & MAP_LOAD)) row = map_block(g, row);
          R.v[b][r][e] = (LDP == LD_L2) ? ld_l2(in + row + n) : ld_stream(in + row + n);
        }
      } else if constexpr (SMEM_A) {
        float4 raw = sm[n * 8 + bc[b]];
        const Chunk<C, VW> ch = *reinterpret_cast<const Chunk<C, VW>*>(&raw);
#pragma unroll
        for (int e = 0; e < VW; ++e) R.v[b][r][e] = ch.v[e];
      } else if ((EXT & EXT_BS) && (g.bs_mode & BS_LOAD_MOD)) {
        // element-wise: a row of x has bs_L points (any alignment)
        const int64_t mask = ((int64_t)1 << g.bs_logM) - 1;
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          const int64_t vo = bin + bc[b] * VW + e + (int64_t)n * g.sn_in;
          const int64_t p = vo & mask;
          C x = p < g.bs_L ? ld_stream(in + (vo >> g.bs_logM) * g.bs_L + p) : C{0, 0};
          const C w = p < g.bs_L ? ld_tw(chirp + p) : C{0, 0};
          if (g.conj_in) x.y = -x.y;
          R.v[b][r][e] = cmul(x, w);
        }
      } else {
        int64_t off = bin + bc[b] * VW + (int64_t)n * g.sn_in;
        if ((EXT & EXT_MAP) && (g.map_mode & MAP_LOAD)) off = map_block(g, off);  // a chunk stays contiguous
        const void* src = in + off;
        float4 raw = (LDP == LD_L2)  ? __ldcg(reinterpret_cast<const float4*>(src))
                     : (FETCH == 256) ? ld_chunk_256(src)
                                      : ld_chunk(src);
        const Chunk<C, VW> ch = *reinterpret_cast<const Chunk<C, VW>*>(&raw);
#pragma unroll
        for (int e = 0; e < VW; ++e) R.v[b][r][e] = ch.v[e];
      }
    }
  }
}

// Phases A (first radix stage of the loaded inputs in R), B and C of tile
// `tile`: everything after the loads.
template <typename T, int L, int R0, int R1, int R2, int NT, bool IN_ROW, int LDP_, int STP_, bool DISCARD_,
          bool SMEM_A = false, int EXT = 0>
__device__ __forceinline__ void fast_finish(const PassGeom& g, const typename Cx<T>::type* in,
                                            typename Cx<T>::type* out,
                                            const PassTables<typename Cx<T>::type>& tb, int64_t tile,
                                            float4* sm, FastRegs<T, L, R0, R1, R2, NT>& R, TilePolicy pol) {
  using C = typename Cx<T>::type;
  const int STP = (STP_ == POLICY_RUNTIME) ? pol.st : STP_;
  const bool DISCARD = (LDP_ == POLICY_RUNTIME) ? (pol.discard != 0) : DISCARD_;
  using Cfg = FastCfg<L, R0, R1, R2, NT>;
  constexpr int VW = ChunkT<T>::VW;
  constexpr int W = 8 * VW;
  constexpr int S = Cfg::S;
  constexpr int RL = (S == 3) ? R2 : R1;  // radix of the last stage
  constexpr bool SW = !SMEM_A;
  static_assert(!(SMEM_A && IN_ROW), "shared-memory input is a column tile");

  const int tid = threadIdx.x;
  const FastTileAt at = fast_tile_at<W>(g, tile);
  const int64_t w0 = at.w0, bin = at.bin, bout = at.bout, tconst = at.tconst;

  // ---------------- phase A: radix-R0 stage of the loaded inputs ----------------
  {
    constexpr int M0 = L / R0;  // stride between the inputs of one butterfly
    auto& v = R.v;
    int bj[Cfg::NB0], bc[Cfg::NB0];
#pragma unroll
    for (int b = 0; b < Cfg::NB0; ++b) fast_butterfly<L, R0, NT, IN_ROW>(b, bj[b], bc[b]);
#pragma unroll
    for (int b = 0; b < Cfg::NB0; ++b) {
#pragma unroll
      for (int e = 0; e < VW; ++e) {
        C x[R0];
#pragma unroll
        for (int r = 0; r < R0; ++r) {
          x[r] = v[b][r][e];
          if (g.conj_in && !((EXT & EXT_BS) && (g.bs_mode & BS_LOAD_MOD))) x[r].y = -x[r].y;  // the fused load conjugates
        }
        dft<R0>(x);
        if (bj[b] != 0) {
#pragma unroll
          for (int r = 1; r < R0; ++r) x[r] = cmul(x[r], ld_tw(tb.twL + bj[b] * r));
        }
#pragma unroll
        for (int r = 0; r < R0; ++r) v[b][r][e] = x[r];
      }
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        Chunk<C, VW> ch;
#pragma unroll
        for (int e = 0; e < VW; ++e) ch.v[e] = v[b][r][e];
        const int p = bj[b] + r * M0;
        sm[sidx<SW>(p, bc[b])] = *reinterpret_cast<float4*>(&ch);
      }
    }
  }
  __syncthreads();
  if (DISCARD) {
    // every input line of this tile has been consumed: W rows (IN_ROW) of L
    // points, or L rows of one 128-byte column chunk
    constexpr int LINE = 128 / (int)sizeof(C);
    if constexpr (IN_ROW) {
      constexpr int LPR = L / LINE;  // lines per input row
      for (int l = tid; l < W * LPR; l += NT)
        discard_line(in + bin + (int64_t)(l / LPR) * g.sin[0] + (l % LPR) * LINE);
    } else {
      for (int l = tid; l < L; l += NT) discard_line(in + bin + (int64_t)l * g.sn_in);
    }
  }

  // ---------------- phase B: middle stage (3-stage plans) ----------------
  if constexpr (S == 3) {
    constexpr int SPAN = L / R0;
    constexpr int M1 = SPAN / R1;
#pragma unroll
    for (int b = 0; b < Cfg::NB1; ++b) {
      const int id = tid + b * NT;
      const int c = id & 7;
      const int q = id >> 3;  // [0, L/R1)
      const int blk = q / M1, j = q % M1;
      const int base = blk * SPAN + j;
      C x[R1][VW];
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        float4 raw = sm[sidx<SW>(base + r * M1, c)];
        const Chunk<C, VW> ch = *reinterpret_cast<const Chunk<C, VW>*>(&raw);
#pragma unroll
        for (int e = 0; e < VW; ++e) x[r][e] = ch.v[e];
      }
#pragma unroll
      for (int e = 0; e < VW; ++e) {
        C y[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) y[r] = x[r][e];
        dft<R1>(y);
        if (j != 0) {
#pragma unroll
          for (int r = 1; r < R1; ++r) y[r] = cmul(y[r], ld_tw(tb.twL + j * r * R0));
        }
#pragma unroll
        for (int r = 0; r < R1; ++r) x[r][e] = y[r];
      }
#pragma unroll
      for (int r = 0; r < R1; ++r) {
        Chunk<C, VW> ch;
#pragma unroll
        for (int e = 0; e < VW; ++e) ch.v[e] = x[r][e];
        sm[sidx<SW>(base + r * M1, c)] = *reinterpret_cast<float4*>(&ch);
      }
    }
    __syncthreads();
  }

  // ---------------- phase C: last stage, natural-order store ----------------
  {
    constexpr int NBL = (S == 3) ? Cfg::NB2 : Cfg::NB1;
    const T scale = (T)g.scale;
#pragma unroll
    for (int b = 0; b < NBL; ++b) {
      const int id = tid + b * NT;
      const int c = id & 7;
      const int blk = id >> 3;  // [0, L/RL)
      // digits of blk: 3 stages: blk = d0*R1 + d1 ; 2 stages: blk = d0
      int kbase;
      if constexpr (S == 3) {
        const int d0 = blk / R1, d1 = blk % R1;
        kbase = d0 + R0 * d1;
      } else {
        kbase = blk;
      }
      constexpr int KSTRIDE = L / RL;  // output stride of the last digit
      C x[RL][VW];
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        float4 raw = sm[sidx<SW>(blk * RL + r, c)];
        const Chunk<C, VW> ch = *reinterpret_cast<const Chunk<C, VW>*>(&raw);
#pragma unroll
        for (int e = 0; e < VW; ++e) x[r][e] = ch.v[e];
      }
#pragma unroll
      for (int e = 0; e < VW; ++e) {
        C y[RL];
#pragma unroll
        for (int r = 0; r < RL; ++r) y[r] = x[r][e];
        dft<RL>(y);
#pragma unroll
        for (int r = 0; r < RL; ++r) x[r][e] = y[r];
      }
      // four-step twiddle w_N^{k t} over this thread's outputs k = kbase +
      // r*KSTRIDE: a running product twc *= w_N^{KSTRIDE t}, taken afresh
      // from the two-level table every kTwAnchor outputs, so each element
      // needs (2 + 2*RL/kTwAnchor)/RL table reads instead of 2 (the reads
      // are scattered when t differs per lane) and carries at most
      // kTwAnchor - 1 extra roundings.
      constexpr int kTwAnchor = 4;
      C twc[VW], tws[VW];
      int64_t tcol[VW];
      if (g.tw_mode == TW_POST) {
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          tcol[e] = (g.tw_dim == 0) ? (w0 + c * VW + e) : tconst;
          const int64_t ms = (int64_t)KSTRIDE * tcol[e];
          tws[e] = cmul(ld_tw(tb.tw_hi + (ms >> g.tw_shift)), ld_tw(tb.tw_lo + (ms & g.tw_mask)));
        }
      }
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int k = kbase + r * KSTRIDE;
        Chunk<C, VW> ch;
#pragma unroll
        for (int e = 0; e < VW; ++e) {
          C y = x[r][e];
          if (g.tw_mode == TW_POST) {
            if (r % kTwAnchor == 0) {
              const int64_t m = (int64_t)k * tcol[e];
              twc[e] = cmul(ld_tw(tb.tw_hi + (m >> g.tw_shift)), ld_tw(tb.tw_lo + (m & g.tw_mask)));
            } else {
              twc[e] = cmul(twc[e], tws[e]);
            }
            y = cmul(y, twc[e]);
          }
          if ((EXT & EXT_BS) && (g.bs_mode & (BS_STORE_MULH | BS_STORE_DEMOD))) {
            const int64_t vo = bout + c * VW + e + (int64_t)k * g.sk_out;
            const int64_t p = vo & (((int64_t)1 << g.bs_logM) - 1);
            if (g.bs_mode & BS_STORE_MULH) {
              y = cmul(y, ld_tw(tb.bs_H + p));
              y.y = -y.y;
            } else {
              if (p < g.bs_L) {
                C a = y;
                a.y = -a.y;
                C r = cmul(ld_tw(tb.bs_chirp + p), a);
                r.x *= scale;
                r.y *= scale;
                if (g.conj_out) r.y = -r.y;
                out[(vo >> g.bs_logM) * g.bs_L + p] = r;
              }
              continue;
            }
          }
          if (g.scale != 1.0) y = cscale(y, scale);
          if (g.conj_out) y.y = -y.y;
          ch.v[e] = y;
        }
        if ((EXT & EXT_BS) && (g.bs_mode & BS_STORE_DEMOD)) continue;  // stored element-wise above
        int64_t off = bout + c * VW + (int64_t)k * g.sk_out;
        if ((EXT & EXT_MAP) && (g.map_mode & MAP_STORE)) off = map_block(g, off);  // a chunk stays contiguous
        float4* dstp = reinterpret_cast<float4*>(out + off);
        if (STP == ST_STREAM)
          st_chunk(dstp, *reinterpret_cast<float4*>(&ch));
        else
          *dstp = *reinterpret_cast<float4*>(&ch);
      }
    }
  }
}

// SMEM_A (column tiles only): the input tile is already in `sm` as dense
// 128-byte rows (row p = input point p); phase A transforms it in place.
template <typename T, int L, int R0, int R1, int R2, int NT, bool IN_ROW, int LDP_, int STP_, bool DISCARD_,
          bool SMEM_A = false, int EXT = 0>
__device__ __forceinline__ void fast_tile(const PassGeom& g, const typename Cx<T>::type* in,
                                          typename Cx<T>::type* out,
                                          const PassTables<typename Cx<T>::type>& tb, int64_t tile,
                                          float4* sm, TilePolicy pol = TilePolicy{0, 0, 0}) {
  const int LDP = (LDP_ == POLICY_RUNTIME) ? pol.ld : LDP_;
  FastRegs<T, L, R0, R1, R2, NT> R;
  fast_load<T, L, R0, R1, R2, NT, IN_ROW, SMEM_A, EXT>(g, in, tile, sm, LDP, R, tb.bs_chirp);
  fast_finish<T, L, R0, R1, R2, NT, IN_ROW, LDP_, STP_, DISCARD_, SMEM_A, EXT>(g, in, out, tb, tile, sm, R, pol);
}

// EXT: the plain pass (0), or the instantiation with the fused Bluestein
// loads and stores (EXT_BS) or with an exchange block map (EXT_MAP)
template <typename T, int L, int R0, int R1, int R2, int NT, bool IN_ROW, int EXT = 0>
__global__ void __launch_bounds__(NT)
    k_fft_fast(const __grid_constant__ PassGeom g, const typename Cx<T>::type* in,
               typename Cx<T>::type* out, const __grid_constant__ PassTables<typename Cx<T>::type> tb) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  fast_tile<T, L, R0, R1, R2, NT, IN_ROW, LD_STREAM, ST_STREAM, false, false, EXT>(
      g, in, out, tb, blockIdx.x, reinterpret_cast<float4*>(smem_raw));
}

// Ask L2 for every input line of tile `tile` (one prefetch per 128-byte
// line; the same lines the tile's loads read, so only valid tiles).  bulk
// (row tiles): one bulk asynchronous prefetch per row (cp.async.bulk.
// prefetch.L2, L points from a 16-byte aligned row start; rows that do not
// start on 16 bytes take the per-line prefetches).
template <typename T, int L, int NT, bool IN_ROW>
__device__ __forceinline__ void fast_prefetch(const PassGeom& g, const typename Cx<T>::type* in, int64_t tile,
                                              bool bulk) {
  using C = typename Cx<T>::type;
  constexpr int W = 8 * ChunkT<T>::VW;
  constexpr int LINE = 128 / (int)sizeof(C);
  const int64_t bin = fast_tile_at<W>(g, tile).bin;
  if constexpr (IN_ROW) {
    constexpr int LPR = L / LINE;  // lines per input row
    static_assert(LPR >= 1, "a row tile covers whole lines");
    static_assert((L * sizeof(C)) % 16 == 0, "a bulk prefetch moves whole 16-byte units");
    if (bulk) {
      static_assert(W <= NT, "one thread per row");
      if (threadIdx.x < W) {
        const C* row = in + bin + (int64_t)threadIdx.x * g.sin[0];
        if ((reinterpret_cast<uintptr_t>(row) & 15) == 0) {
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(row), "r"((int)(L * sizeof(C)))
                       : "memory");
        } else {
          for (int l = 0; l < LPR; ++l) asm volatile("prefetch.global.L2 [%0];" ::"l"(row + l * LINE));
        }
      }
      return;
    }
    for (int l = threadIdx.x; l < W * LPR; l += NT)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(in + bin + (int64_t)(l / LPR) * g.sin[0] + (l % LPR) * LINE));
  } else {
    for (int l = threadIdx.x; l < L; l += NT)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(in + bin + (int64_t)l * g.sn_in));
  }
}

// k_fft_fast with an L2 prefetch of the tile `ahead` tiles on (about one
// wave of resident CTAs later; row tiles by default as one bulk asynchronous
// prefetch per row), issued just before this tile's own loads (so that no
// loaded data is live meanwhile).  The prefetches hold no registers, so the
// SM has more reads in flight than three tiles' worth of loads alone.  Same
// arithmetic and results as k_fft_fast.
// (Resident CTAs per SM it is compiled for: the occupancy the plain kernel
// reaches at its own register count, so that the prefetch costs no CTA slot;
// 80 registers for the complex64 512-point pass.)
template <typename T, int L>
constexpr int fast_pf_min_blocks() {
  return sizeof(T) == 4 ? (L <= 256 ? 4 : (L == 512 ? 3 : 1)) : (L <= 256 ? 5 : 2);
}
// FETCH = 256 (column tiles): the tile's own loads ask for 256-byte L2
// fetches; ahead = 0: no prefetch; bulk: row prefetches as bulk copies.
template <typename T, int L, int R0, int R1, int R2, int NT, bool IN_ROW, int FETCH = 0>
__global__ void __launch_bounds__(NT, fast_pf_min_blocks<T, L>())
    k_fft_fast_pf(const __grid_constant__ PassGeom g, const typename Cx<T>::type* in,
                  typename Cx<T>::type* out, const __grid_constant__ PassTables<typename Cx<T>::type> tb,
                  int64_t ahead, int bulk) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float4* sm = reinterpret_cast<float4*>(smem_raw);
  const int64_t nt = (int64_t)blockIdx.x + ahead;
  if (ahead > 0 && nt < g.ntiles) fast_prefetch<T, L, NT, IN_ROW>(g, in, nt, bulk != 0);
  FastRegs<T, L, R0, R1, R2, NT> R;
  fast_load<T, L, R0, R1, R2, NT, IN_ROW, false, 0, FETCH>(g, in, blockIdx.x, sm, LD_STREAM, R);
  fast_finish<T, L, R0, R1, R2, NT, IN_ROW, LD_STREAM, ST_STREAM, false>(g, in, out, tb, blockIdx.x, sm, R,
                                                                         TilePolicy{0, 0, 0});
}

// Two axes of a stack of square L x L planes in one HBM pass, as a
// persistent dataflow kernel.  Control words (zeroed before each launch):
// 64-bit ticket counter at ctl[0..1], error flag ctl[2], per-plane counters
// ctl[4 + plane].  Work items ("tickets", claimed in increasing order) are
// the X tiles of plane g followed by the Y tiles of plane g - lag:
//   X tile : row tiles of `src` -> transposed column tiles of `mid` (default
//            L2 policy: the plane is read back moments later), then the
//            plane's counter ctl[4 + plane] is incremented (after a gpu fence);
//   Y tile : waits until that counter reaches the plane's X-tile count, then
//            reads row tiles of `mid` at L2 -> natural-order column tiles of
//            `dst`, and discards the consumed `mid` lines from L2 so the
//            intermediate never reaches HBM.
// Only about lag + (resident CTAs / tiles per plane) planes are in flight, so
// their intermediates (2 MiB per 512^2 complex64 plane) stay inside L2.
// Progress: every X ticket of a plane precedes every Y ticket of that plane,
// X items never wait, and a ticket is only claimed by a running CTA, so each
// wait ends.  The wait is still bounded: after kFlowSpinLimit polls the CTA
// sets ctl[2] = 1 (reported by the host as an error) and continues.
// mid must not alias src or dst; src may alias dst.
constexpr unsigned kFlowSpinLimit = 1u << 22;

struct FlowShape {
  int64_t planes, tx, ty, lag;
  TilePolicy xpol, ypol;  // cache policies of the X and Y tiles
};

// ticket -> (is_y, plane, tile within plane); returns false past the end
__device__ __forceinline__ bool flow_decode(const FlowShape& f, int64_t t, bool& is_y, int64_t& plane,
                                            int64_t& tile) {
  const int64_t P = f.planes, D = f.lag, tx = f.tx, ty = f.ty;
  const int64_t A = D * tx, Bm = (P - D) * (tx + ty);
  if (t < A) {
    is_y = false;
    plane = t / tx;
    tile = t % tx;
    return true;
  }
  if (t < A + Bm) {
    const int64_t u = t - A, g = D + u / (tx + ty), r = u % (tx + ty);
    if (r < tx) {
      is_y = false;
      plane = g;
      tile = r;
    } else {
      is_y = true;
      plane = g - D;
      tile = r - tx;
    }
    return true;
  }
  const int64_t u = t - A - Bm;
  if (u >= D * ty) return false;
  is_y = true;
  plane = P - D + u / ty;
  tile = u % ty;
  return true;
}

template <typename T, int L, int R0, int R1, int R2, int NT>
__global__ void __launch_bounds__(NT, (L * 128 <= 64 * 1024) ? 3 : 1)
    k_fft_plane_flow(const __grid_constant__ PassGeom gx, const __grid_constant__ PassGeom gy,
                     const typename Cx<T>::type* src, typename Cx<T>::type* mid,
                     typename Cx<T>::type* dst,
                     const __grid_constant__ PassTables<typename Cx<T>::type> tb, int* ctl,
                     const FlowShape f) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float4* sm = reinterpret_cast<float4*>(smem_raw);
  // two ticket slots after the tile (dynamic shared memory is L*128 + 128 bytes)
  volatile long long* s_tk = reinterpret_cast<volatile long long*>(smem_raw + L * 128);
  unsigned long long* ticket = reinterpret_cast<unsigned long long*>(ctl);
  if (threadIdx.x == 0) s_tk[0] = (long long)atomicAdd(ticket, 1ull);
  __syncthreads();
  for (int slot = 0;; slot ^= 1) {
    const int64_t t = s_tk[slot];
    // claim the next ticket now; it is published by this item's last barrier
    if (threadIdx.x == 0) s_tk[slot ^ 1] = (long long)atomicAdd(ticket, 1ull);
    bool is_y;
    int64_t plane, tile;
    if (!flow_decode(f, t, is_y, plane, tile)) break;
    if (!is_y) {
      fast_tile<T, L, R0, R1, R2, NT, true, POLICY_RUNTIME, POLICY_RUNTIME, false>(
          gx, src, mid, tb, plane * f.tx + tile, sm, f.xpol);
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctl + 4 + plane, 1);
      }
    } else {
      if (threadIdx.x == 0) {
        unsigned it = 0;
        for (;;) {
          int v;
          asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(ctl + 4 + plane) : "memory");
          if (v >= f.tx) break;
          if (++it > kFlowSpinLimit) {
            atomicExch(ctl + 2, 1);
            break;
          }
          __nanosleep(64);
        }
      }
      __syncthreads();
      fast_tile<T, L, R0, R1, R2, NT, true, POLICY_RUNTIME, POLICY_RUNTIME, false>(
          gy, mid, dst, tb, plane * f.ty + tile, sm, f.ypol);
      __syncthreads();
    }
  }
}

}  // namespace shafft_sm100
