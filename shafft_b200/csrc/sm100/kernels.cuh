// Device kernels of the sm_100a C2C FFT backend.
//
// k_fft_pass  -- one HBM pass: batched length-L DFTs on W-wide tiles.
//   Phase 1: each thread loads the R inputs of a first-stage butterfly
//            straight from HBM (coalesced: lanes walk b0 for column tiles or
//            n for row tiles), applies input conjugation / four-step
//            pre-twiddle, runs the radix-R butterfly in registers, applies
//            the decimation-in-frequency twiddle and writes the R results to
//            shared memory in place.
//   Phase 2: the remaining radix stages run in shared memory, in place
//            (Cooley-Tukey DIF; span shrinks by the stage radix).  The
//            shared tile is [L][W] with an odd row pitch (W+1), so 16 lanes
//            that share a row and differ in w never hit the same bank, and
//            16 lanes that walk rows with a fixed w do not either.
//   Phase 3: results are read back in digit-reversed order through a small
//            permutation table and stored to HBM with the four-step
//            post-twiddle, scale and output conjugation fused in.
// The same source serves a runtime length (LS == 0) and compile-time
// specialisations for the hot lengths, where all index arithmetic folds.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "butterflies.cuh"
#include "pass.h"

namespace shafft_sm100 {

template <typename C>
__device__ __forceinline__ C tw_n(const PassTables<C>& tb, int shift, int64_t mask, int64_t m) {
  C hi = tb.tw_hi[m >> shift];
  C lo = tb.tw_lo[m & mask];
  return cmul(hi, lo);
}

template <int R, typename C>
__device__ __forceinline__ void stage_first(const PassGeom& g, const PassTables<C>& tb, const C* in,
                                            C* sm, int L, int W, int logW, int pitch, int nst,
                                            int wcount, int64_t bin, int64_t w0, int64_t tconst) {
  const int m0 = L / R;
  const int nbf = m0 << logW;
  for (int b = threadIdx.x; b < nbf; b += kThreads) {
    int w, j;
    if (g.in_row) {
      j = b % m0;
      w = b / m0;
    } else {
      w = b & (W - 1);
      j = b >> logW;
    }
    const bool valid = w < wcount;
    const C* src = in + bin + (int64_t)w * g.sin[0];
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int n = j + r * m0;
      C x = valid ? src[(int64_t)n * g.sn_in] : C{0, 0};
      if (g.conj_in) x.y = -x.y;
      if (g.tw_mode == TW_PRE) {
        const int64_t t = (g.tw_dim == 0) ? (w0 + w) : tconst;
        x = cmul(x, tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)n * t));
      }
      v[r] = x;
    }
    dft<R>(v);
    if (nst > 1 && j != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tb.twL[j * r]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) sm[(j + r * m0) * pitch + w] = v[r];
  }
}

template <int R, typename C>
__device__ __forceinline__ void stage_mid(const PassTables<C>& tb, C* sm, int L, int W, int logW,
                                          int pitch, int span, int Ls) {
  const int m = span / R;
  const int nbf = (L / R) << logW;
  for (int b = threadIdx.x; b < nbf; b += kThreads) {
    const int w = b & (W - 1);
    const int q = b >> logW;
    const int blk = q / m;
    const int j = q - blk * m;
    const int base = blk * span + j;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = sm[(base + r * m) * pitch + w];
    dft<R>(v);
    if (m > 1 && j != 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tb.twL[j * r * Ls]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) sm[(base + r * m) * pitch + w] = v[r];
  }
}

#define SHAFFT_RADIX_DISPATCH(RAD, CALL) \
  switch (RAD) {                         \
    case 2: CALL(2); break;              \
    case 3: CALL(3); break;              \
    case 4: CALL(4); break;              \
    case 5: CALL(5); break;              \
    case 7: CALL(7); break;              \
    case 8: CALL(8); break;              \
    case 11: CALL(11); break;            \
    case 13: CALL(13); break;            \
    case 16: CALL(16); break;            \
    default: break;                      \
  }

__host__ __device__ constexpr int ilog2c(int x) {
  int l = 0;
  while ((1 << l) < x) ++l;
  return l;
}

// One output of a direct-DFT tile, with the pass's fused post-twiddle,
// scale and output conjugation.
template <typename T, typename C>
__device__ __forceinline__ void direct_put(const PassGeom& g, const PassTables<C>& tb, C* out, C y, int k, int w,
                                           int64_t bout, int64_t w0, int64_t tconst, T scale) {
  if (g.tw_mode == TW_POST) {
    const int64_t tt = (g.tw_dim == 0) ? (w0 + w) : tconst;
    y = cmul(y, tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)k * tt));
  }
  if (g.scale != 1.0) y = cscale(y, scale);
  if (g.conj_out) y.y = -y.y;
  out[bout + (int64_t)w * g.sout[0] + (int64_t)k * g.sk_out] = y;
}

// Direct DFT of the tile held in shared memory (natural order, [n][w] with
// the given pitch), X[k] = sum_n x[n] w^{nk} with w = exp(-2 pi i / L),
// evaluated in pairs.  With s[n] = x[n] + x[L-n] and d[n] = x[n] - x[L-n]
// for n = 1 .. h (h = (L-1)/2), and e_k = (-1)^k x[L/2] for even L (0 for
// odd L):
//   X[k]   = x[0] + e_k + sum_n s[n] Re w^{nk} + i sum_n d[n] Im w^{nk}
//   X[L-k] = x[0] + e_k + sum_n s[n] Re w^{nk} - i sum_n d[n] Im w^{nk}
// for k = 1 .. h; X[0] = x[0] + sum_n s[n] + x[L/2] and, for even L,
// X[L/2] = x[0] + sum_n (-1)^n s[n] + (-1)^{L/2} x[L/2].  Each table read
// and each pair of real multiplies then serves two outputs, a quarter of
// the arithmetic of the plain sum; the exponent n*k is reduced modulo L
// incrementally.  Used for lengths with a prime factor above 13 when L is
// small enough that O(L) work per output beats a Bluestein round trip.
// Outputs go straight to HBM with the pass's fused twiddle/scale/conj.
template <typename T, typename C>
__device__ __forceinline__ void direct_store(const PassGeom& g, const PassTables<C>& tb, C* sm, C* out, int L,
                                             int W, int logW, int pitch, int wcount, int64_t bout, int64_t w0,
                                             int64_t tconst) {
  const int h = (L - 1) / 2;
  const bool even = (L & 1) == 0;
  // s and d in place: row n <- s[n], row L-n <- d[n]
  for (int b = threadIdx.x; b < (h << logW); b += kThreads) {
    const int w = b & (W - 1), n = 1 + (b >> logW);
    const C a = sm[n * pitch + w], c = sm[(L - n) * pitch + w];
    sm[n * pitch + w] = C{a.x + c.x, a.y + c.y};
    sm[(L - n) * pitch + w] = C{a.x - c.x, a.y - c.y};
  }
  __syncthreads();
  const T scale = (T)g.scale;
  // item (j, w): j = 0 gives X[0] (and X[L/2] for even L), j = 1 .. h gives
  // X[j] and X[L-j]
  const int items = (h + 1) << logW;
  for (int b = threadIdx.x; b < items; b += kThreads) {
    const int w = b & (W - 1), j = b >> logW;
    if (w >= wcount) continue;
    const C x0 = sm[w];
    const C xh = even ? sm[(L / 2) * pitch + w] : C{0, 0};
    if (j == 0) {
      C y0 = x0, yh = x0;
      T sg = -1;
      for (int n = 1; n <= h; ++n) {
        const C sn = sm[n * pitch + w];
        y0.x += sn.x;
        y0.y += sn.y;
        yh.x += sg * sn.x;
        yh.y += sg * sn.y;
        sg = -sg;
      }
      y0.x += xh.x;
      y0.y += xh.y;
      direct_put<T, C>(g, tb, out, y0, 0, w, bout, w0, tconst, scale);
      if (even) {
        const T e = ((L / 2) & 1) ? (T)-1 : (T)1;
        yh.x += e * xh.x;
        yh.y += e * xh.y;
        direct_put<T, C>(g, tb, out, yh, L / 2, w, bout, w0, tconst, scale);
      }
      continue;
    }
    T px = 0, py = 0, qx = 0, qy = 0;
    int m = 0;
    for (int n = 1; n <= h; ++n) {
      m += j;
      if (m >= L) m -= L;
      const C t = tb.twL[m];
      const C sn = sm[n * pitch + w], dn = sm[(L - n) * pitch + w];
      px += sn.x * t.x;
      py += sn.y * t.x;
      qx += dn.x * t.y;
      qy += dn.y * t.y;
    }
    const T e = (j & 1) ? (T)-1 : (T)1;
    const T bx = x0.x + e * xh.x + px, by = x0.y + e * xh.y + py;
    direct_put<T, C>(g, tb, out, C{bx - qy, by + qx}, j, w, bout, w0, tconst, scale);
    direct_put<T, C>(g, tb, out, C{bx + qy, by - qx}, L - j, w, bout, w0, tconst, scale);
  }
}

// One W-wide tile of a generic pass (runtime length and radix list; nst == 0
// selects the direct DFT).  `sm` holds L * pitch elements.
template <typename T, int LS, int WS>
__device__ __forceinline__ void generic_tile(const PassGeom& g, const typename Cx<T>::type* in,
                                             typename Cx<T>::type* out,
                                             const PassTables<typename Cx<T>::type>& tb, int64_t tile,
                                             typename Cx<T>::type* sm) {
  using C = typename Cx<T>::type;
  constexpr RadixPlan P = radix_plan(LS > 0 ? LS : 1);
  const int L = LS ? LS : g.L;
  const int W = WS ? WS : g.W;
  const int logW = WS ? ilog2c(WS) : g.logW;
  const int pitch = g.pitch;  // generic_pitch(W, in_row), set by the planner
  const int nst = LS ? P.n : g.nst;

  int64_t rest = tile;
  const int64_t tw = rest % g.tiles_w;
  rest /= g.tiles_w;
  const int64_t i1 = rest % g.ext[1];
  rest /= g.ext[1];
  const int64_t i2 = rest % g.ext[2];
  const int64_t i3 = rest / g.ext[2];
  const int64_t w0 = tw * W;
  const int wcount = (int)((g.ext[0] - w0) < W ? (g.ext[0] - w0) : W);
  const int64_t bin = w0 * g.sin[0] + i1 * g.sin[1] + i2 * g.sin[2] + i3 * g.sin[3];
  const int64_t bout = w0 * g.sout[0] + i1 * g.sout[1] + i2 * g.sout[2] + i3 * g.sout[3];
  const int64_t tconst = g.tw_dim == 1 ? i1 : (g.tw_dim == 2 ? i2 : (g.tw_dim == 3 ? i3 : 0));

  if (!LS && nst == 0) {
    // direct DFT: load the tile in natural order, then O(L) per output
    const int total = L << logW;
    for (int b = threadIdx.x; b < total; b += kThreads) {
      int w, n;
      if (g.in_row) {
        n = b % L;
        w = b / L;
      } else {
        w = b & (W - 1);
        n = b >> logW;
      }
      C x = (w < wcount) ? in[bin + (int64_t)w * g.sin[0] + (int64_t)n * g.sn_in] : C{0, 0};
      if (g.conj_in) x.y = -x.y;
      if (g.tw_mode == TW_PRE) {
        const int64_t t = (g.tw_dim == 0) ? (w0 + w) : tconst;
        x = cmul(x, tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)n * t));
      }
      sm[n * pitch + w] = x;
    }
    __syncthreads();
    direct_store<T, C>(g, tb, sm, out, L, W, logW, pitch, wcount, bout, w0, tconst);
    return;
  }

  // phase 1: load + first radix stage
  {
    const int r0 = LS ? P.r[0] : g.rad[0];
#define SHAFFT_CALL_FIRST(R) \
  stage_first<R, C>(g, tb, in, sm, L, W, logW, pitch, nst, wcount, bin, w0, tconst)
    SHAFFT_RADIX_DISPATCH(r0, SHAFFT_CALL_FIRST)
#undef SHAFFT_CALL_FIRST
  }
  __syncthreads();
  // phase 2: remaining stages in shared memory
  {
    int span = L;
#pragma unroll
    for (int s = 1; s < (LS ? P.n : kMaxStages); ++s) {
      if (!LS && s >= nst) break;
      span /= (LS ? P.r[s - 1] : g.rad[s - 1]);
      const int Ls = L / span;
      const int rs = LS ? P.r[s] : g.rad[s];
#define SHAFFT_CALL_MID(R) stage_mid<R, C>(tb, sm, L, W, logW, pitch, span, Ls)
      SHAFFT_RADIX_DISPATCH(rs, SHAFFT_CALL_MID)
#undef SHAFFT_CALL_MID
      __syncthreads();
    }
  }
  // phase 3: digit-reversed read, fused twiddle/scale/conj, store
  const int total = L << logW;
  const T scale = (T)g.scale;
  if (g.out_row) {
    for (int b = threadIdx.x; b < total; b += kThreads) {
      const int k = b % L, w = b / L;
      if (w >= wcount) continue;
      C x = sm[tb.k2p[k] * pitch + w];
      if (g.tw_mode == TW_POST) {
        const int64_t t = (g.tw_dim == 0) ? (w0 + w) : tconst;
        x = cmul(x, tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)k * t));
      }
      if (g.scale != 1.0) x = cscale(x, scale);
      if (g.conj_out) x.y = -x.y;
      out[bout + (int64_t)w * g.sout[0] + (int64_t)k * g.sk_out] = x;
    }
  } else {
    // column output walked in natural k order: a thread keeps its column
    // w = tid mod W (W divides kThreads) and visits k = k0, k0 + KS, ...
    // (KS = kThreads / W), so the four-step twiddle w_N^{k t} is a running
    // product by w_N^{KS t}, taken afresh from the table every 4 outputs
    // (the table reads are scattered across the lanes)
    const int KS = kThreads >> logW;
    const int w = threadIdx.x & (W - 1);
    const bool tw = g.tw_mode == TW_POST && w < wcount;
    const int64_t t = (g.tw_dim == 0) ? (w0 + w) : tconst;
    C tstep = C{1, 0}, tcur = C{1, 0};
    if (tw && KS < L) tstep = tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)KS * t);
    int i = 0;
    for (int b = threadIdx.x; b < total; b += kThreads, ++i) {
      if (w >= wcount) continue;
      const int k = b >> logW;
      C x = sm[tb.k2p[k] * pitch + w];
      if (tw) {
        tcur = (i % 4 == 0) ? tw_n(tb, g.tw_shift, g.tw_mask, (int64_t)k * t) : cmul(tcur, tstep);
        x = cmul(x, tcur);
      }
      if (g.scale != 1.0) x = cscale(x, scale);
      if (g.conj_out) x.y = -x.y;
      out[bout + (int64_t)w * g.sout[0] + (int64_t)k * g.sk_out] = x;
    }
  }
}

template <typename T, int LS, int WS>
__global__ void __launch_bounds__(kThreads)
    k_fft_pass(const __grid_constant__ PassGeom g, const typename Cx<T>::type* in,
               typename Cx<T>::type* out, const __grid_constant__ PassTables<typename Cx<T>::type> tb) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  for (int64_t tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
    generic_tile<T, LS, WS>(g, in, out, tb, tile, sm);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------

// data[i] = conj?(src[i]) * factor   (normalize, copies)
template <typename T>
__global__ void k_scale_copy(const typename Cx<T>::type* src, typename Cx<T>::type* dst, int64_t n,
                             T factor, int conj) {
  using C = typename Cx<T>::type;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    C x = src[i];
    x.x *= factor;
    x.y *= factor;
    if (conj) x.y = -x.y;
    dst[i] = x;
  }
}

// The Bluestein element-wise steps run on a 2-D grid: blockIdx.y walks the
// batch rows b = o*I + i (one division per row), blockIdx.x/threadIdx.x the
// points of a row in block tiles of kEwUnroll*blockDim points, each thread
// loading its kEwUnroll points before it computes (independent loads in
// flight; the arrays are L2-resident at the lengths Bluestein pads to).
constexpr int kEwUnroll = 4;

// Bluestein modulate: dst[b*M + m] = (m < L) ? conj?(x(o, m, i)) * chirp[m] : 0
// with b = o*I + i and x(o, m, i) = src[(o*L + m)*I + i].
template <typename T>
__global__ void k_bs_modulate(const typename Cx<T>::type* src, typename Cx<T>::type* dst, int64_t L,
                              int64_t M, int64_t I, int64_t rows, const typename Cx<T>::type* chirp,
                              int conj) {
  using C = typename Cx<T>::type;
  const int64_t tile = (int64_t)blockDim.x * kEwUnroll;
  for (int64_t b = blockIdx.y; b < rows; b += gridDim.y) {
    const int64_t o = b / I, i = b - o * I;
    const C* srow = src + o * L * I + i;
    C* drow = dst + b * M;
    for (int64_t base = blockIdx.x * tile + threadIdx.x; base < M; base += gridDim.x * tile) {
      C x[kEwUnroll], w[kEwUnroll];
#pragma unroll
      for (int u = 0; u < kEwUnroll; ++u) {
        const int64_t m = base + (int64_t)u * blockDim.x;
        x[u] = m < L ? srow[m * I] : C{0, 0};
        w[u] = m < L ? chirp[m] : C{0, 0};
      }
#pragma unroll
      for (int u = 0; u < kEwUnroll; ++u) {
        const int64_t m = base + (int64_t)u * blockDim.x;
        if (conj) x[u].y = -x[u].y;
        if (m < M) drow[m] = cmul(x[u], w[u]);
      }
    }
  }
}

// s[b*M + m] = conj(s[b*M + m] * H[m])   (H carries the 1/M of the inverse)
template <typename T>
__global__ void k_bs_mulh(typename Cx<T>::type* s, const typename Cx<T>::type* H, int64_t M,
                          int64_t rows) {
  using C = typename Cx<T>::type;
  const int64_t tile = (int64_t)blockDim.x * kEwUnroll;
  for (int64_t b = blockIdx.y; b < rows; b += gridDim.y) {
    C* row = s + b * M;
    for (int64_t base = blockIdx.x * tile + threadIdx.x; base < M; base += gridDim.x * tile) {
      C x[kEwUnroll], h[kEwUnroll];
#pragma unroll
      for (int u = 0; u < kEwUnroll; ++u) {
        const int64_t m = base + (int64_t)u * blockDim.x;
        x[u] = m < M ? row[m] : C{0, 0};
        h[u] = m < M ? H[m] : C{0, 0};
      }
#pragma unroll
      for (int u = 0; u < kEwUnroll; ++u) {
        const int64_t m = base + (int64_t)u * blockDim.x;
        C y = cmul(x[u], h[u]);
        y.y = -y.y;
        if (m < M) row[m] = y;
      }
    }
  }
}

// Bluestein demodulate: dst(o, k, i) = conj?(chirp[k] * conj(s[b*M + k])) * scale
template <typename T>
__global__ void k_bs_demod(const typename Cx<T>::type* s, typename Cx<T>::type* dst, int64_t L,
                           int64_t M, int64_t I, int64_t rows, const typename Cx<T>::type* chirp,
                           int conj, T scale) {
  using C = typename Cx<T>::type;
  const int64_t tile = (int64_t)blockDim.x * kEwUnroll;
  for (int64_t b = blockIdx.y; b < rows; b += gridDim.y) {
    const int64_t o = b / I, i = b - o * I;
    const C* srow = s + b * M;
    C* drow = dst + o * L * I + i;
    for (int64_t base = blockIdx.x * tile + threadIdx.x; base < L; base += gridDim.x * tile) {
      C v[kEwUnroll], w[kEwUnroll];
#pragma unroll
      for (int u = 0; u < kEwUnroll; ++u) {
        const int64_t k = base + (int64_t)u * blockDim.x;
        v[u] = k < L ? srow[k] : C{0, 0};
        w[u] = k < L ? chirp[k] : C{0, 0};
      }
#pragma unroll
      for (int u = 0; u < kEwUnroll; ++u) {
        const int64_t k = base + (int64_t)u * blockDim.x;
        C a = v[u];
        a.y = -a.y;
        C r = cmul(w[u], a);
        r.x *= scale;
        r.y *= scale;
        if (conj) r.y = -r.y;
        if (k < L) drow[k * I] = r;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Table generation (FP64 phase, rounded once to the storage type)
// ---------------------------------------------------------------------------

// out[i] = exp(-2*pi*i * ((i*mult) mod N) / N), i < count
template <typename T>
__global__ void k_gen_twiddle(typename Cx<T>::type* out, int64_t count, int64_t mult, int64_t N) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t m = ((unsigned __int128)(uint64_t)i * (uint64_t)mult) % (uint64_t)N;
    double s, c;
    sincospi(-2.0 * ((double)m / (double)N), &s, &c);
    out[i] = typename Cx<T>::type{(T)c, (T)s};
  }
}

// chirp[m] = exp(-i*pi*(m^2 mod 2L)/L), m < L  (integer phase reduction)
template <typename T>
__global__ void k_gen_chirp(typename Cx<T>::type* out, int64_t L) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < L;
       m += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t r = ((unsigned __int128)(uint64_t)m * (uint64_t)m) % (uint64_t)(2 * L);
    double s, c;
    sincospi(-((double)r / (double)L), &s, &c);
    out[m] = typename Cx<T>::type{(T)c, (T)s};
  }
}

// Bluestein kernel sequence h (length M): conj(chirp[|j|]) cyclically, zero elsewhere.
template <typename T>
__global__ void k_gen_bs_kernel(typename Cx<T>::type* h, const typename Cx<T>::type* chirp, int64_t L,
                                int64_t M) {
  using C = typename Cx<T>::type;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < M;
       j += (int64_t)gridDim.x * blockDim.x) {
    C r = C{0, 0};
    if (j < L) {
      r = chirp[j];
      r.y = -r.y;
    } else if (j > M - L) {
      r = chirp[M - j];
      r.y = -r.y;
    }
    h[j] = r;
  }
}

}  // namespace shafft_sm100
