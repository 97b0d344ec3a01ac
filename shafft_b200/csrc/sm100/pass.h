// Pass descriptors shared by the host planner (plan.cu) and the device
// kernels (kernels.cu).
//
// A "pass" is one kernel launch that reads the whole working tensor from HBM
// once and writes it once.  It performs batched DFTs of length L (L <= 4096)
// along one logical index "n" of a strided view of the tensor:
//
//   input  element (n, b0, b1, b2, b3) at  in  + n*sn_in  + sum_d b_d*sin[d]
//   output element (k, b0, b1, b2, b3) at  out + k*sk_out + sum_d b_d*sout[d]
//
// b0 is the tile dimension: one CTA processes W consecutive b0 values for one
// (b1, b2, b3) tuple, so every load/store instruction of a warp touches W
// consecutive elements when sin[0]/sout[0] == 1 ("column" orientation) or L
// consecutive elements when sn_in/sk_out == 1 ("row" orientation).
//
// Optional extras fused into the same pass:
//   * a four-step twiddle  w_N^{(n or k) * t}  with t = b_{tw_dim} (applied to
//     the input (PRE) or to the output (POST)); the planner guarantees the
//     exponent is < N so no modular reduction is needed;
//   * conjugation on input / output (backward transforms are computed as
//     conj(F(conj(x))));
//   * a real scale on output (fused normalisation).
#pragma once
#include <stdint.h>

namespace shafft_sm100 {

constexpr int kMaxStages = 16;
constexpr int kMaxPassLen = 4096;
constexpr int kThreads = 256;

enum TwMode : int { TW_NONE = 0, TW_PRE = 1, TW_POST = 2 };

struct RadixPlan {
  int n = 0;
  int r[kMaxStages] = {};
};

// Radix sequence for a pass of length L (L must factor into 2,3,5,7,11,13).
// Powers of two are split into as many 8/16 stages as keep the stage count
// minimal (512 = 8*8*8, 4096 = 16*16*16); odd primes follow.
__host__ __device__ constexpr RadixPlan radix_plan(int L) {
  RadixPlan p{};
  int e = 0;
  while (L % 2 == 0) {
    L /= 2;
    ++e;
  }
  int n16 = e / 4, rem = e % 4;
  int pw[kMaxStages] = {};
  int np = 0;
  if (rem == 0) {
    for (int i = 0; i < n16; ++i) pw[np++] = 16;
  } else if (rem == 3) {
    for (int i = 0; i < n16; ++i) pw[np++] = 16;
    pw[np++] = 8;
  } else if (rem == 2) {
    if (n16 >= 1) {
      for (int i = 0; i < n16 - 1; ++i) pw[np++] = 16;
      pw[np++] = 8;
      pw[np++] = 8;
    } else {
      pw[np++] = 4;
    }
  } else {  // rem == 1
    if (n16 >= 2) {
      for (int i = 0; i < n16 - 2; ++i) pw[np++] = 16;
      pw[np++] = 8;
      pw[np++] = 8;
      pw[np++] = 8;
    } else if (n16 == 1) {
      pw[np++] = 8;
      pw[np++] = 4;
    } else {
      pw[np++] = 2;
    }
  }
  for (int i = 0; i < np; ++i) p.r[p.n++] = pw[i];
  const int odd[5] = {3, 5, 7, 11, 13};
  for (int oi = 0; oi < 5; ++oi)
    while (L % odd[oi] == 0) {
      L /= odd[oi];
      p.r[p.n++] = odd[oi];
    }
  if (L != 1) p.n = -1;  // not representable
  return p;
}

struct PassGeom {
  int L;
  int nst;
  int rad[kMaxStages];
  int W;       // tile width along b0 (power of two)
  int logW;
  int pitch;   // shared-memory row pitch in elements: element (p, w) at p*pitch + w
  int in_row;  // 1: lanes walk n at load (sn_in == 1)
  int out_row; // 1: lanes walk k at store (sk_out == 1)
  int64_t ext[4];
  int64_t sin[4];
  int64_t sout[4];
  int64_t sn_in, sk_out;
  int64_t tiles_w;  // ceil(ext[0] / W)
  int64_t ntiles;   // tiles_w * ext[1] * ext[2] * ext[3]
  int tw_mode;
  int tw_dim;
  int tw_shift;     // two-level table split: m = (m >> shift, m & mask)
  int64_t tw_mask;
  int conj_in, conj_out;
  double scale;
  // Bluestein steps fused into a specialised pass (bits; 0 = none):
  //   BS_LOAD_MOD    load x (rows of bs_L, stride 1) into the virtual rows of
  //                  2^bs_logM points: conj_in(x[p]) * chirp[p] for p < bs_L,
  //                  0 beyond (replaces the modulate step before the pass);
  //   BS_STORE_MULH  store conj(y * H[p]) (the spectrum multiply after it);
  //   BS_STORE_DEMOD store conj_out(chirp[p] * conj(y) * scale) to rows of
  //                  bs_L points, p < bs_L only (the demodulate after it);
  // p is the point's position in its virtual row of 2^bs_logM points.
  int bs_mode;
  int bs_logM;
  int64_t bs_L;
  // Block map of a slab / pencil exchange fused into a specialised pass
  // (bits; 0 = none): the pass reads its input (MAP_LOAD) or writes its
  // output (MAP_STORE) in the per-peer block layout of the row-major array
  // [map_outer][2^map_log_n][2^map_log_inner] instead of the natural layout,
  // for an even partition of the n axis into blocks of 2^map_log_q: natural
  // index v = (o*n + k)*inner + i lives in the block layout at
  //   ((p*map_outer + o)*q + k % q)*inner + i,  p = k / q.
  int map_mode;
  int map_log_n, map_log_inner, map_log_q;
  int64_t map_outer;
};

enum BsMode : int { BS_LOAD_MOD = 1, BS_STORE_MULH = 2, BS_STORE_DEMOD = 4 };
enum MapMode : int { MAP_LOAD = 1, MAP_STORE = 2 };

// Shared-memory row pitch (elements) of a generic-pass tile [L][pitch] whose
// rows hold W columns.  Column-input passes put the W columns of a row on
// consecutive lanes, so a pitch of W keeps their half-warps of 8-byte
// accesses on distinct banks.  Row-input passes put consecutive rows on
// consecutive lanes: with W >= 8 a pitch of W would put a half-warp on one
// bank pair, so they get the odd pitch W + 1; with W <= 4 the conflict is at
// most 4-way and the smaller tile wins.  Measured on B200 against W + 1
// everywhere, FFT1D 1,488,375 fwd+bwd (W = 4): complex64 0.091 -> 0.083 ms,
// complex128 0.152 -> 0.115 ms, the batched form unchanged; W everywhere
// cost the batched form (row passes up to W = 32) 3%.
__host__ __device__ constexpr int generic_pitch(int W, bool in_row) {
  return W == 1 ? 1 : ((in_row && W >= 8) ? W + 1 : W);
}

// Device pointers a pass reads besides its input/output.
template <typename C>
struct PassTables {
  const C* twL;            // w_L^m, m < L
  const uint16_t* p2k;     // digit-reversed position -> frequency index
  const uint16_t* k2p;     // frequency index -> position
  const C* tw_hi;          // w_N^{(m >> shift) << shift}
  const C* tw_lo;          // w_N^{m & mask}
  const void* tcB;         // tensor-core passes: split DFT matrix in shared-memory layout
  const C* bs_chirp;       // Bluestein fused into the pass (PassGeom::bs_mode)
  const C* bs_H;
};

}  // namespace shafft_sm100
