// Real-to-complex and complex-to-real transforms (an extension: the
// reference supports C2C / Z2Z only, docs/limitations.dox:51-60).
//
// A real tensor of dims (d_0, ..., d_{n-1}) with an even last length L is
// read as a complex tensor z of dims (d_0, ..., L/2), z[j] = x[2j] + i x[2j+1]
// along the last axis, at no cost (the same bytes).  Forward (R2C):
//   1. C2C of length L/2 along the last axis:      Z = DFT_{L/2}(z)
//   2. untangle, per row, for k = 0 .. L/2:
//        E[k] = (Z[k] + conj(Z[L/2-k])) / 2       (DFT of the even samples)
//        O[k] = (Z[k] - conj(Z[L/2-k])) / (2i)    (DFT of the odd samples)
//        X[k] = E[k] + w_L^k O[k]                 (Z[L/2] taken as Z[0])
//   3. C2C along every other axis of the (..., L/2 + 1) half spectrum.
// Backward (C2R) runs the steps in reverse, with the untangle inverted:
//        Z[k] = (X[k] + conj(X[L/2-k])) + i w_L^{-k} (X[k] - conj(X[L/2-k]))
// (the Hermitian extension X[k + L/2] = conj(X[L/2 - k]) folded in), and a
// backward C2C of length L/2 whose complex output, read as reals, is the
// unnormalised real inverse y[n] = sum over all L frequencies of the
// Hermitian spectrum.  The output of R2C is the first L/2 + 1 frequencies
// of the last axis (the others follow by Hermitian symmetry), the layout
// FFTW and cuFFT use.  Normalisation (`scale`) is fused into the last step.
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

// forward untangle: Z (rows x H) -> X (rows x (H + 1)), H = L / 2;
// tw[k] = w_L^k (forward sign), k <= H
template <typename T>
__global__ void k_r2c_untangle(const typename Cx<T>::type* Z, typename Cx<T>::type* X, int64_t rows,
                               int64_t H, const typename Cx<T>::type* tw, T scale) {
  using C = typename Cx<T>::type;
  const int64_t total = rows * (H + 1);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / (H + 1), k = i - r * (H + 1);
    const C a = Z[r * H + (k == H ? 0 : k)];
    const C b = cconj(Z[r * H + (k == 0 ? 0 : H - k)]);
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
                             const typename Cx<T>::type* tw) {
  using C = typename Cx<T>::type;
  const int64_t total = rows * H;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / H, k = i - r * H;
    const C a = X[r * (H + 1) + k];
    const C b = cconj(X[r * (H + 1) + (H - k)]);  // X[k + H] by Hermitian symmetry
    const C s = cadd(a, b), d = csub(a, b);
    // i * conj(w_L^k) * d
    const C wd = cmul(d, cconj(tw[k]));
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
  int ndim = 0;
  int64_t rows = 0, H = 0;  // rows of the last axis, L / 2
  shafft_sm100_plan last = nullptr;  // C2C of length H along the last axis of (..., H)
  shafft_sm100_plan rest = nullptr;  // C2C along the other axes of (..., H + 1), or null
  void* tw = nullptr;                // w_L^k, k <= H
  void* a = nullptr;                 // rows x H
  void* b = nullptr;                 // rows x (H + 1), when rest exists
};

namespace {

void rplan_free(shafft_sm100_rplan_s* p) {
  if (p->last) shafft_sm100_plan_destroy(p->last);
  if (p->rest) shafft_sm100_plan_destroy(p->rest);
  if (p->tw) dev_free(p->tw);
  if (p->a) dev_free(p->a);
  if (p->b) dev_free(p->b);
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
  p->ndim = ndim;
  p->H = L / 2;
  p->rows = 1;
  for (int a = 0; a + 1 < ndim; ++a) p->rows *= dims[a];
  const size_t es = precision ? 16 : 8;
  std::vector<int64_t> half(dims, dims + ndim), spec(dims, dims + ndim);
  half[ndim - 1] = p->H;
  spec[ndim - 1] = p->H + 1;
  const int last_axis = ndim - 1;
  int rc = shafft_sm100_plan_create_axes(&p->last, ndim, half.data(), precision, 0, 1, &last_axis);
  if (!rc && ndim > 1) {
    std::vector<int> axes;
    for (int a = 0; a + 1 < ndim; ++a) axes.push_back(a);
    rc = shafft_sm100_plan_create_axes(&p->rest, ndim, spec.data(), precision, 0, (int)axes.size(), axes.data());
  }
  if (rc) {
    rplan_free(p);
    return rc;
  }
  cudaError_t e = dev_malloc(&p->tw, (size_t)(p->H + 1) * es);
  if (e == cudaSuccess) e = dev_malloc(&p->a, (size_t)(p->rows * p->H) * es);
  if (e == cudaSuccess && p->rest) e = dev_malloc(&p->b, (size_t)(p->rows * (p->H + 1)) * es);
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
  int rc = shafft_sm100_execute(p->last, real_in, p->a, 0, 1.0, stream);
  if (rc) return rc;
  void* untangled = p->rest ? p->b : spec_out;
  const double sc = p->rest ? 1.0 : scale;
  const unsigned g = grid_for(p->rows * (p->H + 1));
  if (p->precision)
    k_r2c_untangle<double><<<g, 256, 0, s>>>(reinterpret_cast<const double2*>(p->a),
                                             reinterpret_cast<double2*>(untangled), p->rows, p->H,
                                             reinterpret_cast<const double2*>(p->tw), sc);
  else
    k_r2c_untangle<float><<<g, 256, 0, s>>>(reinterpret_cast<const float2*>(p->a),
                                            reinterpret_cast<float2*>(untangled), p->rows, p->H,
                                            reinterpret_cast<const float2*>(p->tw), (float)sc);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rfail(SHAFFT_SM100_ECUDA, "untangle launch: %s", cudaGetErrorString(e));
  if (p->rest) return shafft_sm100_execute(p->rest, p->b, spec_out, 0, scale, stream);
  return 0;
}

int shafft_sm100_execute_c2r(shafft_sm100_rplan p, void* spec_in, void* real_out, double scale, void* stream) {
  if (!p || !spec_in || !real_out) return rfail(SHAFFT_SM100_EINVAL, "null argument");
  if (real_out == spec_in) return rfail(SHAFFT_SM100_EINVAL, "input and output must be distinct buffers");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const void* spectrum = spec_in;
  if (p->rest) {
    const int rc = shafft_sm100_execute(p->rest, spec_in, p->b, 1, 1.0, stream);
    if (rc) return rc;
    spectrum = p->b;
  }
  const unsigned g = grid_for(p->rows * p->H);
  if (p->precision)
    k_c2r_tangle<double><<<g, 256, 0, s>>>(reinterpret_cast<const double2*>(spectrum),
                                           reinterpret_cast<double2*>(p->a), p->rows, p->H,
                                           reinterpret_cast<const double2*>(p->tw));
  else
    k_c2r_tangle<float><<<g, 256, 0, s>>>(reinterpret_cast<const float2*>(spectrum),
                                          reinterpret_cast<float2*>(p->a), p->rows, p->H,
                                          reinterpret_cast<const float2*>(p->tw));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rfail(SHAFFT_SM100_ECUDA, "tangle launch: %s", cudaGetErrorString(e));
  return shafft_sm100_execute(p->last, p->a, real_out, 1, scale, stream);
}

}  // extern "C"
