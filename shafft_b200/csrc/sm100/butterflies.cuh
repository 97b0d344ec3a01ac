// Register-resident DFT butterflies for the sm_100a FFT passes.
//
// dft<R>(v) overwrites v[0..R) with its forward DFT, V[k] = sum_n v[n] w^{nk},
// w = exp(-2*pi*i/R), natural order in and out.  The backward transform is
// obtained by the passes through conjugation at load and store, so only the
// forward sign is compiled.  Radix 4/8/16 are built from radix-2/4 with the
// Cooley-Tukey split n = n1 + N1*n2, k = N2*k1 + k2; odd primes use the
// symmetric-pair form that needs (p-1)^2/2 real multiply-adds per component.
#pragma once
#include <cuda_runtime.h>

#include "trig_constants.h"

namespace shafft_sm100 {

template <typename T>
struct Cx;
template <>
struct Cx<float> {
  using type = float2;
};
template <>
struct Cx<double> {
  using type = double2;
};

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  return C{a.x + b.x, a.y + b.y};
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  return C{a.x - b.x, a.y - b.y};
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C>
__device__ __forceinline__ C cconj(C a) {
  return C{a.x, -a.y};
}
// multiply by -i
template <typename C>
__device__ __forceinline__ C cmul_mi(C a) {
  return C{a.y, -a.x};
}
template <typename C, typename T>
__device__ __forceinline__ C cscale(C a, T s) {
  return C{a.x * s, a.y * s};
}

// multiply by w_R^m = exp(-2*pi*i*m/R) with compile-time R, m
template <int R, int M, typename C>
__device__ __forceinline__ C ctw(C a) {
  using T = decltype(a.x);
  constexpr int m = ((M % R) + R) % R;
  if constexpr (m == 0) {
    return a;
  } else if constexpr (4 * m == R) {
    return cmul_mi(a);
  } else if constexpr (2 * m == R) {
    return C{-a.x, -a.y};
  } else if constexpr (4 * m == 3 * R) {
    return C{-a.y, a.x};
  } else if constexpr (8 * m == R) {
    constexpr T h = (T)7.071067811865475244008e-1;
    return C{(a.x + a.y) * h, (a.y - a.x) * h};
  } else if constexpr (8 * m == 3 * R) {
    constexpr T h = (T)7.071067811865475244008e-1;
    return C{(a.y - a.x) * h, -(a.x + a.y) * h};
  } else {
    constexpr T c = (T)trig_cos(R, m);
    constexpr T s = (T)trig_sin(R, m);
    // (x + iy)(c - is)
    return C{a.x * c + a.y * s, a.y * c - a.x * s};
  }
}

template <typename C>
__device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <typename C>
__device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3) {
  C a0 = cadd(x0, x2), a1 = csub(x0, x2);
  C a2 = cadd(x1, x3), a3 = cmul_mi(csub(x1, x3));
  x0 = cadd(a0, a2);
  x2 = csub(a0, a2);
  x1 = cadd(a1, a3);
  x3 = csub(a1, a3);
}

template <typename C>
__device__ __forceinline__ void dft8(C* v) {
  // even/odd split: E = DFT4(v0,v2,v4,v6), O = DFT4(v1,v3,v5,v7)
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3);
  dft4(o0, o1, o2, o3);
  o1 = ctw<8, 1>(o1);
  o2 = ctw<8, 2>(o2);
  o3 = ctw<8, 3>(o3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

template <typename C>
__device__ __forceinline__ void dft16(C* v) {
  // n = n1 + 4*n2; inner DFT4 over n2 per n1, twiddle w16^{n1*k2},
  // outer DFT4 over n1 per k2 -> X[4*k1 + k2]
  C y[16];
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
    C a = v[n1], b = v[n1 + 4], c = v[n1 + 8], d = v[n1 + 12];
    dft4(a, b, c, d);
    y[n1 * 4 + 0] = a;
    y[n1 * 4 + 1] = b;
    y[n1 * 4 + 2] = c;
    y[n1 * 4 + 3] = d;
  }
  y[1 * 4 + 1] = ctw<16, 1>(y[1 * 4 + 1]);
  y[1 * 4 + 2] = ctw<16, 2>(y[1 * 4 + 2]);
  y[1 * 4 + 3] = ctw<16, 3>(y[1 * 4 + 3]);
  y[2 * 4 + 1] = ctw<16, 2>(y[2 * 4 + 1]);
  y[2 * 4 + 2] = ctw<16, 4>(y[2 * 4 + 2]);
  y[2 * 4 + 3] = ctw<16, 6>(y[2 * 4 + 3]);
  y[3 * 4 + 1] = ctw<16, 3>(y[3 * 4 + 1]);
  y[3 * 4 + 2] = ctw<16, 6>(y[3 * 4 + 2]);
  y[3 * 4 + 3] = ctw<16, 9>(y[3 * 4 + 3]);
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    C a = y[0 * 4 + k2], b = y[1 * 4 + k2], c = y[2 * 4 + k2], d = y[3 * 4 + k2];
    dft4(a, b, c, d);
    v[0 + k2] = a;
    v[4 + k2] = b;
    v[8 + k2] = c;
    v[12 + k2] = d;
  }
}

// 32 points: DFT16 of the even and the odd points, then one radix-2 stage
// with the twiddles w32^k: X[k] = E[k] + w^k O[k], X[k+16] = E[k] - w^k O[k]
template <int K, typename C>
__device__ __forceinline__ void dft32_combine(C* v, const C* e, const C* o) {
  if constexpr (K < 16) {
    const C t = ctw<32, K>(o[K]);
    v[K] = cadd(e[K], t);
    v[K + 16] = csub(e[K], t);
    dft32_combine<K + 1>(v, e, o);
  }
}

template <typename C>
__device__ __forceinline__ void dft32(C* v) {
  C e[16], o[16];
#pragma unroll
  for (int n = 0; n < 16; ++n) {
    e[n] = v[2 * n];
    o[n] = v[2 * n + 1];
  }
  dft16(e);
  dft16(o);
  dft32_combine<0>(v, e, o);
}

// odd prime p: X_0 = x_0 + sum_j a_j, and for k = 1..(p-1)/2
//   X_k     = x_0 + sum_j a_j cos(2 pi jk/p) - i sum_j b_j sin(2 pi jk/p)
//   X_{p-k} = x_0 + sum_j a_j cos(2 pi jk/p) + i sum_j b_j sin(2 pi jk/p)
// with a_j = x_j + x_{p-j}, b_j = x_j - x_{p-j}.
template <int P, typename C>
__device__ __forceinline__ void dft_odd(C* v) {
  using T = decltype(v[0].x);
  constexpr int H = (P - 1) / 2;
  C a[H], b[H];
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    a[j - 1] = cadd(v[j], v[P - j]);
    b[j - 1] = csub(v[j], v[P - j]);
  }
  C x0 = v[0];
  C s0 = x0;
#pragma unroll
  for (int j = 0; j < H; ++j) s0 = cadd(s0, a[j]);
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    C re = x0, im = C{0, 0};
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      const T c = (T)trig_cos(P, (j * k) % P);
      const T s = (T)trig_sin(P, (j * k) % P);
      re.x += a[j - 1].x * c;
      re.y += a[j - 1].y * c;
      im.x += b[j - 1].x * s;
      im.y += b[j - 1].y * s;
    }
    // -i * im = (im.y, -im.x)
    v[k] = C{re.x + im.y, re.y - im.x};
    v[P - k] = C{re.x - im.y, re.y + im.x};
  }
  v[0] = s0;
}

template <int R, typename C>
__device__ __forceinline__ void dft(C* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8(v);
  } else if constexpr (R == 16) {
    dft16(v);
  } else if constexpr (R == 32) {
    dft32(v);
  } else {
    static_assert(R == 3 || R == 5 || R == 7 || R == 11 || R == 13, "unsupported radix");
    dft_odd<R>(v);
  }
}

}  // namespace shafft_sm100
