// Real-to-complex and complex-to-real transforms (an extension: the
// reference supports C2C / Z2Z only, docs/limitations.dox:51-60).
//
// A real tensor of dims (d_0, ..., d_{n-1}) with an even last length L is
// read as a complex tensor z of dims (d_0, ..., L/2), z[.., j] = x[.., 2j] +
// i x[.., 2j+1], at no cost (the same bytes).  With H = L/2, J the index over
// the other axes and -J its mirror (every other index negated modulo its
// length), forward (R2C):
//   1. the C2C transform of z over every axis (the library's ordinary plan
//      of dims (d_0, ..., H): its specialised passes apply): Z = DFT(z)
//   2. untangle, for k = 0 .. H (Z[J, H] taken as Z[J, 0]):
//        E = (Z[J, k] + conj(Z[-J, H-k])) / 2     (spectrum of the even samples)
//        O = (Z[J, k] - conj(Z[-J, H-k])) / (2i)  (spectrum of the odd samples)
//        X[J, k] = E + w_L^k O
// Backward (C2R) inverts the untangle with the Hermitian extension
// X[J, k + H] = conj(X[-J, H - k]) folded in,
//        Z[J, k] = (X[J, k] + conj(X[-J, H-k])) + i w_L^{-k} (X[J, k] - conj(X[-J, H-k])),
// then runs the backward C2C of z, whose complex output read as reals is the
// unnormalised real inverse.  The R2C output is the first H + 1 frequencies
// of the last axis (the others follow by Hermitian symmetry), the layout FFTW
// and cuFFT use.  Normalisation (`scale`) is fused into the last step.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <new>
#include <vector>

#include "../../../include/shafft_sm100.h"
#include "butterflies.cuh"
#include "launch.h"

namespace shafft_sm100 {
namespace {

int rfail(int code, const char* fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof(msg), fmt, ap);
  va_end(ap);
  return report_error(code, msg);
}

// Other axes of the tensor (all but the last): lengths and row-major
// strides, for the mirror index -J.
struct RDims {
  int n;
  int64_t len[16];
  int64_t stride[16];
};

__device__ __forceinline__ int64_t mirror_row(const RDims& d, int64_t row) {
  int64_t m = 0;
  for (int a = d.n - 1; a >= 0; --a) {
    const int64_t j = row % d.len[a];
    row /= d.len[a];
    m += (j ? d.len[a] - j : 0) * d.stride[a];
  }
  return m;
}

// forward untangle: Z (rows x H) -> X (rows x (H + 1)), H = L / 2;
// tw[k] = w_L^k (forward sign), k <= H
template <typename T>
__global__ void k_r2c_untangle(const typename Cx<T>::type* Z, typename Cx<T>::type* X, int64_t rows,
                               int64_t H, const typename Cx<T>::type* tw, T scale, const RDims d) {
  using C = typename Cx<T>::type;
  const int64_t total = rows * (H + 1);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / (H + 1), k = i - r * (H + 1);
    const int64_t mr = mirror_row(d, r);
    const C a = Z[r * H + (k == H ? 0 : k)];
    const C b = cconj(Z[mr * H + (k == 0 ? 0 : H - k)]);
    const C e = C{(a.x + b.x) * (T)0.5, (a.y + b.y) * (T)0.5};
    // (a - b) / (2i) = (a.y - b.y, -(a.x - b.x)) / 2
    const C o = C{(a.y - b.y) * (T)0.5, (b.x - a.x) * (T)0.5};
    C x = cadd(e, cmul(o, tw[k]));
    if (scale != (T)1) x = cscale(x, scale);
    X[i] = x;
  }
}

// backward untangle: X (rows x (H + 1)) -> Z (rows x H)
template <typename T>
__global__ void k_c2r_tangle(const typename Cx<T>::type* X, typename Cx<T>::type* Z, int64_t rows, int64_t H,
                             const typename Cx<T>::type* tw, const RDims d) {
  using C = typename Cx<T>::type;
  const int64_t total = rows * H;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / H, k = i - r * H;
    const int64_t mr = mirror_row(d, r);
    const C a = X[r * (H + 1) + k];
    const C b = cconj(X[mr * (H + 1) + (H - k)]);  // X[J, k + H] by Hermitian symmetry
    const C s = cadd(a, b), dd = csub(a, b);
    // i * conj(w_L^k) * dd
    const C wd = cmul(dd, cconj(tw[k]));
    Z[i] = C{s.x - wd.y, s.y + wd.x};
  }
}

template <typename T>
__global__ void k_r2c_twiddle(typename Cx<T>::type* tw, int64_t L) {
  const int64_t H = L / 2;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= H; k += (int64_t)gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)L, &s, &c);
    tw[k] = typename Cx<T>::type{(T)c, (T)s};
  }
}

unsigned grid_for(int64_t n) {
  const int64_t g = (n + 255) / 256;
  return (unsigned)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace
}  // namespace shafft_sm100

using namespace shafft_sm100;

struct shafft_sm100_rplan_s {
  int precision = 0;
  int64_t rows = 0, H = 0;        // rows of the last axis, L / 2
  shafft_sm100_plan full = nullptr;  // C2C over every axis of (..., H)
  RDims dims{};                   // the other axes, for the mirror index
  void* tw = nullptr;             // w_L^k, k <= H
  void* a = nullptr;              // rows x H
};

namespace {

void rplan_free(shafft_sm100_rplan_s* p) {
  if (p->full) shafft_sm100_plan_destroy(p->full);
  if (p->tw) dev_free(p->tw);
  if (p->a) dev_free(p->a);
  delete p;
}

}  // namespace

extern "C" {

int shafft_sm100_rplan_create(shafft_sm100_rplan* out, int ndim, const int64_t* dims, int precision) {
  if (!out || !dims || ndim < 1 || ndim > 16) return rfail(SHAFFT_SM100_EINVAL, "bad real-transform arguments");
  if (precision != 0 && precision != 1) return rfail(SHAFFT_SM100_EINVAL, "bad precision");
  *out = nullptr;
  for (int a = 0; a < ndim; ++a)
    if (dims[a] < 1) return rfail(SHAFFT_SM100_EINVAL, "axis %d has length %lld", a, (long long)dims[a]);
  const int64_t L = dims[ndim - 1];
  if (L % 2) return rfail(SHAFFT_SM100_ENOTSUP, "the last axis (%lld) must have an even length", (long long)L);
  auto* p = new (std::nothrow) shafft_sm100_rplan_s();
  if (!p) return rfail(SHAFFT_SM100_EALLOC, "host allocation failed");
  p->precision = precision;
  p->H = L / 2;
  p->rows = 1;
  p->dims.n = ndim - 1;
  for (int a = ndim - 2; a >= 0; --a) {
    p->dims.len[a] = dims[a];
    p->dims.stride[a] = p->rows;
    p->rows *= dims[a];
  }
  const size_t es = precision ? 16 : 8;
  std::vector<int64_t> half(dims, dims + ndim);
  half[ndim - 1] = p->H;
  int rc = shafft_sm100_plan_create_nd(&p->full, ndim, half.data(), precision);
  if (rc) {
    p->full = nullptr;
    rplan_free(p);
    return rc;
  }
  cudaError_t e = dev_malloc(&p->tw, (size_t)(p->H + 1) * es);
  if (e == cudaSuccess) e = dev_malloc(&p->a, (size_t)(p->rows * p->H) * es);
  if (e != cudaSuccess) {
    cudaGetLastError();
    rplan_free(p);
    return rfail(SHAFFT_SM100_EALLOC, "device allocation for the real transform failed");
  }
  if (precision)
    k_r2c_twiddle<double><<<grid_for(p->H + 1), 256>>>(reinterpret_cast<double2*>(p->tw), L);
  else
    k_r2c_twiddle<float><<<grid_for(p->H + 1), 256>>>(reinterpret_cast<float2*>(p->tw), L);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
  if (e != cudaSuccess) {
    rplan_free(p);
    return rfail(SHAFFT_SM100_ECUDA, "real-transform twiddles: %s", cudaGetErrorString(e));
  }
  *out = p;
  return 0;
}

int shafft_sm100_rplan_destroy(shafft_sm100_rplan p) {
  if (p) rplan_free(p);
  return 0;
}

int64_t shafft_sm100_rplan_spectrum_elements(shafft_sm100_rplan p) {
  return p ? p->rows * (p->H + 1) : 0;
}

int shafft_sm100_execute_r2c(shafft_sm100_rplan p, void* real_in, void* spec_out, double scale, void* stream) {
  if (!p || !real_in || !spec_out) return rfail(SHAFFT_SM100_EINVAL, "null argument");
  if (real_in == spec_out) return rfail(SHAFFT_SM100_EINVAL, "input and output must be distinct buffers");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int rc = shafft_sm100_execute(p->full, real_in, p->a, 0, 1.0, stream);
  if (rc) return rc;
  const unsigned g = grid_for(p->rows * (p->H + 1));
  if (p->precision)
    k_r2c_untangle<double><<<g, 256, 0, s>>>(reinterpret_cast<const double2*>(p->a),
                                             reinterpret_cast<double2*>(spec_out), p->rows, p->H,
                                             reinterpret_cast<const double2*>(p->tw), scale, p->dims);
  else
    k_r2c_untangle<float><<<g, 256, 0, s>>>(reinterpret_cast<const float2*>(p->a),
                                            reinterpret_cast<float2*>(spec_out), p->rows, p->H,
                                            reinterpret_cast<const float2*>(p->tw), (float)scale, p->dims);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rfail(SHAFFT_SM100_ECUDA, "untangle launch: %s", cudaGetErrorString(e));
  return 0;
}

int shafft_sm100_execute_c2r(shafft_sm100_rplan p, void* spec_in, void* real_out, double scale, void* stream) {
  if (!p || !spec_in || !real_out) return rfail(SHAFFT_SM100_EINVAL, "null argument");
  if (real_out == spec_in) return rfail(SHAFFT_SM100_EINVAL, "input and output must be distinct buffers");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned g = grid_for(p->rows * p->H);
  if (p->precision)
    k_c2r_tangle<double><<<g, 256, 0, s>>>(reinterpret_cast<const double2*>(spec_in),
                                           reinterpret_cast<double2*>(p->a), p->rows, p->H,
                                           reinterpret_cast<const double2*>(p->tw), p->dims);
  else
    k_c2r_tangle<float><<<g, 256, 0, s>>>(reinterpret_cast<const float2*>(spec_in),
                                          reinterpret_cast<float2*>(p->a), p->rows, p->H,
                                          reinterpret_cast<const float2*>(p->tw), p->dims);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rfail(SHAFFT_SM100_ECUDA, "tangle launch: %s", cudaGetErrorString(e));
  return shafft_sm100_execute(p->full, p->a, real_out, 1, scale, stream);
}

}  // extern "C"
