// Host-side launchers of the device kernels, one explicit instantiation per
// element type (launch_f32.cu, launch_f64.cu), so that the planner in
// plan.cu stays plain host code and the kernel TUs compile in parallel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pass.h"

struct shafft_sm100_plan_s;

namespace shafft_sm100 {

// Record `msg` as this thread's last error of the library (returned by
// shafft_sm100_last_error_message) and return `code`.
int report_error(int code, const char* msg);

// Device allocations of the library (guard.cu): plain cudaMalloc / cudaFree,
// or, with SHAFFT_SM100_CANARY=1, blocks with guard bytes on both sides that
// dev_free checks (a changed guard returns SHAFFT_SM100_ECUDA with a message).
bool guard_enabled();
cudaError_t dev_malloc(void** ptr, size_t bytes);
int dev_free(void* ptr);

// Launches of the bulk-tensor-copy column pass (k_fft_fast_tma) in this
// process (plan.cu).
void count_tma_launch();

// True when executes of `plan` may run at the same time on different
// streams (plan.cu): it has no scratch buffers and no step with per-launch
// control words, so every launch reads only the plan's tables and the
// caller's buffers (its error word is only ever set, by a bounded wait that
// gave up).
bool plan_shareable(const shafft_sm100_plan_s* plan);

// Tensor-core (tcgen05, split FP16) pass for complex64: one DFT stage of
// length 2..64 over every row of the geometry g (tc.cu).  `err` is a device
// int set to 1 when a wait for the tensor core gives up.
bool tc_supported(const PassGeom& g);
size_t tc_smem_bytes(int L);
// bytes of the split DFT matrix of length L, and its generation (FP64 phases,
// FP16 hi/lo split, in the layout k_fft_tc copies into shared memory)
size_t tc_table_bytes(int L);
int tc_gen_table(void* dst, int L, cudaStream_t s);
template <typename C>
struct PassTables;
int tc_pass(const PassGeom& g, const float2* in, float2* out, const PassTables<float2>& tb, int* err,
            cudaStream_t s);

// Two axes of a stack of 512 x 512 complex64 planes in one pass, one 16-CTA
// cluster per plane exchanging through distributed shared memory
// (plane_cluster.cu).  plane_cluster_available() is false on a device that
// cannot co-schedule such clusters; the planner then keeps two passes.
bool plane_cluster_len(int precision, int64_t L);
bool plane_cluster_available();
size_t plane_cluster_smem();
// `err` is a device int set to 1 when a wait for the prefetch copies gives up.
cudaError_t plane_cluster_pass(const float2* in, float2* out, int64_t planes, int64_t pstride_in,
                               int64_t pstride_out, const float2* tw, int conj_in, int conj_out,
                               double scale, int* err, cudaStream_t s);

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

template <typename T>
struct Launch {
  using C = typename Vec2<T>::type;
  // raise the dynamic shared-memory limit of every pass kernel on the
  // current device (idempotent)
  static cudaError_t init();
  // init() once per device and element type: function attributes belong to
  // each device's context, so a process that plans on several devices sets
  // them on every one (thread-safe; later calls return the first result)
  static cudaError_t init_device();
  static cudaError_t pass(const PassGeom& g, const C* in, C* out, const PassTables<C>& tb,
                          size_t smem, cudaStream_t s);
  // specialised pass for a hot length; tile width is 16 bytes x 8 (= 8*VW
  // elements), output is a column tile.  Returns cudaErrorNotSupported when
  // no specialisation exists for L.
  // Column tiles of L = 256 / 512 go through the bulk-tensor-copy kernel
  // (k_fft_fast_tma) when the input qualifies; `err` is its device error word.
  static cudaError_t fast(const PassGeom& g, bool in_row, const C* in, C* out,
                          const PassTables<C>& tb, int* err, cudaStream_t s);
  static bool fast_supported(int L);
  static int fast_threads(int L);
  // L2 prefetch distance (quarter waves of resident CTAs) of the plain
  // specialised pass of length L with row (in_row) or column input; 0 when
  // it runs k_fft_fast without prefetching
  static int fast_prefetch(int L, bool in_row);
  // fused two-axis pass over a stack of square L x L planes (see
  // k_fft_plane_flow); ctl holds 4 + planes ints of plan-owned device memory
  static cudaError_t plane(const PassGeom& gx, const PassGeom& gy, const C* src, C* mid, C* dst,
                           const PassTables<C>& tb, int planes, int* ctl, int lag, cudaStream_t s);
  static bool plane_supported(int L);
  static cudaError_t scale_copy(const C* src, C* dst, int64_t n, T factor, int conj, cudaStream_t s);
  static cudaError_t bs_modulate(const C* src, C* dst, int64_t L, int64_t M, int64_t I,
                                 int64_t total, const C* chirp, int conj, cudaStream_t s);
  static cudaError_t bs_mulh(C* s_, const C* H, int64_t M, int64_t total, cudaStream_t s);
  static cudaError_t bs_demod(const C* src, C* dst, int64_t L, int64_t M, int64_t I, int64_t total,
                              const C* chirp, int conj, T scale, cudaStream_t s);
  static cudaError_t gen_twiddle(C* out, int64_t count, int64_t mult, int64_t N, cudaStream_t s);
  static cudaError_t gen_chirp(C* out, int64_t L, cudaStream_t s);
  static cudaError_t gen_bs_kernel(C* h, const C* chirp, int64_t L, int64_t M, cudaStream_t s);
};

// per-precision specialisations (defined in launch_f32.cu / launch_f64.cu)
template <>
bool Launch<float>::fast_supported(int L);
template <>
bool Launch<double>::fast_supported(int L);
template <>
int Launch<float>::fast_threads(int L);
template <>
int Launch<double>::fast_threads(int L);
template <>
int Launch<float>::fast_prefetch(int L, bool in_row);
template <>
int Launch<double>::fast_prefetch(int L, bool in_row);
template <>
bool Launch<float>::plane_supported(int L);
template <>
bool Launch<double>::plane_supported(int L);
template <>
cudaError_t Launch<float>::plane(const PassGeom& gx, const PassGeom& gy, const float2* src,
                                 float2* mid, float2* dst, const PassTables<float2>& tb, int planes,
                                 int* ctl, int lag, cudaStream_t s);
template <>
cudaError_t Launch<double>::plane(const PassGeom& gx, const PassGeom& gy, const double2* src,
                                  double2* mid, double2* dst, const PassTables<double2>& tb,
                                  int planes, int* ctl, int lag, cudaStream_t s);
template <>
cudaError_t Launch<float>::fast(const PassGeom& g, bool in_row, const float2* in, float2* out,
                                const PassTables<float2>& tb, int* err, cudaStream_t s);
template <>
cudaError_t Launch<double>::fast(const PassGeom& g, bool in_row, const double2* in, double2* out,
                                 const PassTables<double2>& tb, int* err, cudaStream_t s);

extern template struct Launch<float>;
extern template struct Launch<double>;

}  // namespace shafft_sm100
