/*
 * shafft_sm100.h -- C ABI of the B200 (sm_100a) C2C FFT kernel library,
 * libshafft_sm100.so.
 *
 * This is the thin layer the SHAFFT host library (libshafft.so, which keeps
 * the reference's FFTND/FFT1D classes and C API) reaches the CUDA kernels
 * through.  Plain pointers, sizes and int status codes; no exceptions, no
 * C++ or torch types.
 *
 * Each entry point replaces a backend "method" call of the reference
 * (paths relative to the SHAFFT project):
 *   shafft_sm100_plan_create_nd  <- fftndPlan      src/cpp/fft/hipfft_method/fftnd_method.cpp:162-351
 *                                   (hipfftMakePlanMany64 at :323-335)
 *   shafft_sm100_plan_create_1d  <- fft1dPlan      src/cpp/fft/hipfft_method/fft1d_method.hip:416-581
 *   shafft_sm100_execute         <- fftndExecute   src/cpp/fft/hipfft_method/fftnd_method.cpp:371-533
 *                                   (hipfftExecC2C/Z2Z at :486-497) and
 *                                   fft1dExecute   src/cpp/fft/hipfft_method/fft1d_method.hip:628-650
 *   shafft_sm100_scale           <- normalizeComplexFloat/Double
 *                                   src/cpp/fft/hipfft_method/common/normalize.hip:41-77
 *   shafft_sm100_plan_destroy    <- fftndDestroy / fft1dDestroy
 *   shafft_sm100_set_stream      <- fftndSetStream src/cpp/fft/hipfft_method/fftnd_method.cpp:353-369
 *
 * Conventions: row-major, last axis fastest; forward = exp(-2*pi*i*jk/n);
 * execute is unnormalised unless a scale != 1 is passed (the fused
 * normalisation of the last pass).  Element types: precision 0 = complex64
 * (interleaved float re/im), 1 = complex128 (interleaved double).
 *
 * Return codes: 0 success, otherwise one of SHAFFT_SM100_E*.
 */
#ifndef SHAFFT_SM100_H
#define SHAFFT_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHAFFT_SM100_OK 0
#define SHAFFT_SM100_EINVAL 1   /* bad argument (null pointer, size, dims)   */
#define SHAFFT_SM100_EALLOC 2   /* device allocation failed                  */
#define SHAFFT_SM100_ECUDA 3    /* CUDA runtime error (see last_cuda_error)  */
#define SHAFFT_SM100_ENOTSUP 4  /* size outside what the planner can handle  */

typedef struct shafft_sm100_plan_s* shafft_sm100_plan;

/* Plan a C2C transform over every axis of a row-major tensor dims[0..ndim).
 * Builds twiddle / chirp / permutation tables on the current device (FP64
 * generation) and allocates plan-owned scratch when Bluestein stages need it.
 * Synchronous with respect to the host. */
int shafft_sm100_plan_create_nd(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                int precision);

/* Plan flags for shafft_sm100_plan_create_nd_ex / shafft_sm100_plan_query_ex.
 * SHAFFT_SM100_PLAN_TENSOR_CORE: complex64 only.  Every pass of length <= 64
 * runs on the tensor cores (tcgen05 MMA, split FP16 hi/lo operands, FP32
 * accumulation, per-row power-of-two scaling); axes are factored into at
 * most 4 (1-D) or 3 (inner axes) such passes, anything else keeps the plain
 * kernels.  No counterpart in the reference (its GPU path is hipFFT). */
#define SHAFFT_SM100_PLAN_TENSOR_CORE 1
/* SHAFFT_SM100_PLAN_TC_PRIME_AXES: complex64 only.  Tensor-core passes only
 * for axes whose length has a prime factor above 13 (where the plain path
 * computes O(L^2) direct DFTs or Bluestein); every other axis keeps the
 * plain specialised passes.  Ignored when SHAFFT_SM100_PLAN_TENSOR_CORE is
 * also set.  No counterpart in the reference. */
#define SHAFFT_SM100_PLAN_TC_PRIME_AXES 2
/* SHAFFT_SM100_PLAN_MEASURE (or SHAFFT_SM100_PLANNER=MEASURE in the
 * environment, which applies it to every plan): build and time each distinct
 * pass list the planner's choices give for this shape (multi-pass factor
 * splits, generic tile widths, and -- only with
 * SHAFFT_SM100_PLAN_TC_PRIME_AXES -- tensor-core passes or not), keep the
 * fastest, and cache the choice per shape in SHAFFT_SM100_PLAN_CACHE (default
 * ~/.cache/shafft_sm100_plans.txt).  Plan creation then allocates two
 * transform-sized scratch buffers for the duration of the measurement.  The
 * counterpart of the reference's SHAFFT_FFTW_PLANNER=MEASURE. */
#define SHAFFT_SM100_PLAN_MEASURE 4

int shafft_sm100_plan_create_nd_ex(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                   int precision, int flags);

/* Transform only the listed axes of the tensor dims[0..ndim) (the others are
 * batch axes); naxes < 0 or axes == NULL selects every axis.  The per-stage
 * subplans of a slab-decomposed transform use this, as the reference's
 * fftndPlan(nta, ta, ...) does (src/cpp/fft/hipfft_method/fftnd_method.cpp:162-351). */
int shafft_sm100_plan_create_axes(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                  int precision, int flags, int naxes, const int* axes);

/* Like shafft_sm100_plan_create_axes, with a slab / pencil exchange's block
 * packing fused into the plan: load_map / store_map = {outer, n, inner,
 * parts} (NULL or parts = 0: none) say that the input is read from / the
 * output is written to the per-peer block layout of the row-major array
 * [outer][n][inner] (outer * n * inner = the plan's elements): block p,
 * holding indices [start_p, start_p + len_p) of the n axis, is the contiguous
 * segment [outer][len_p][inner] at offset outer * start_p * inner, with the
 * block partition of shafft_sm100_pack_blocks.  A map is fused when n,
 * inner and parts are powers of two (even blocks) and the plan's first step
 * (load) or last step (store) is an out-of-place specialised pass whose
 * accesses stay inside the runs the map keeps contiguous (a block's
 * n / parts * inner elements);
 * *fused returns bit 0 = load map fused, bit 1 = store map fused (a one-step
 * plan takes only the store map).  A map that is not fused is not applied:
 * the caller packs or unpacks with shafft_sm100_pack_blocks /
 * shafft_sm100_unpack_blocks instead.  Replaces the separate pack / unpack
 * of the reference's slab exchange (src/cpp/slab_nd.cpp:23-56, 596-654). */
int shafft_sm100_plan_create_axes_mapped(shafft_sm100_plan* out, int ndim, const int64_t* dims,
                                         int precision, int flags, int naxes, const int* axes,
                                         const int64_t* load_map, const int64_t* store_map, int* fused);
/* The steps such a plan would have, as shafft_sm100_plan_describe JSON with
 * "fused" added (planning only: no device work, callable without a GPU). */
int shafft_sm100_plan_query_mapped(int ndim, const int64_t* dims, int precision, int naxes, const int* axes,
                                   const int64_t* load_map, const int64_t* store_map, char* buf, int buflen);

/* Plan a 1-D C2C transform of length n (equivalent to the 1-D ND plan). */
int shafft_sm100_plan_create_1d(shafft_sm100_plan* out, int64_t n, int precision);

int shafft_sm100_plan_destroy(shafft_sm100_plan plan);

/* Default stream for shafft_sm100_execute calls that pass stream == NULL. */
int shafft_sm100_set_stream(shafft_sm100_plan plan, void* stream /* cudaStream_t */);

/* Execute: src -> dst.  direction 0 = forward, 1 = backward.  The output is
 * multiplied by `scale` (pass 1.0 for the unnormalised transform).  src and
 * dst must be distinct, 16-byte aligned device buffers (cudaMalloc memory
 * is; others return SHAFFT_SM100_EINVAL) of at least plan_elements()
 * complex elements; src's contents are undefined afterwards (it is used as
 * ping-pong space).  Asynchronous: enqueued on `stream` (cudaStream_t; NULL
 * selects the plan's stream). */
int shafft_sm100_execute(shafft_sm100_plan plan, void* src, void* dst, int direction, double scale,
                         void* stream);

/* data[i] *= factor over count complex elements (stand-alone normalize). */
int shafft_sm100_scale(void* data, size_t count, int precision, double factor, void* stream);

/* Status of the plan's last executes: reads the device-side error flags of
 * the passes with bounded waits (tensor-core passes, bulk-copy column passes,
 * the fused plane pass), set if one of those waits gave up.  Call after
 * synchronising the stream; returns 0 or SHAFFT_SM100_ECUDA. */
int shafft_sm100_plan_status(shafft_sm100_plan plan);

/* Column passes launched in this process through the bulk-tensor-copy
 * kernel (length 256 / 512 column tiles; opt-in with SHAFFT_SM100_TMA=1). */
int64_t shafft_sm100_tma_launch_count(void);

/* Number of complex elements of the transform. */
int64_t shafft_sm100_plan_elements(shafft_sm100_plan plan);

/* Number of full HBM passes one execute performs (kernel launches that
 * read and write the whole tensor, counting elementwise Bluestein steps). */
int shafft_sm100_plan_passes(shafft_sm100_plan plan);

/* Number of kernel launches one execute performs. */
int shafft_sm100_plan_launches(shafft_sm100_plan plan);

/* Plan-owned device bytes (tables + scratch). */
size_t shafft_sm100_plan_device_bytes(shafft_sm100_plan plan);

/* Host-only planning query (no device needed): writes a JSON description of
 * the pass list for the given shape into buf.  Returns the status code. */
int shafft_sm100_plan_query(int ndim, const int64_t* dims, int precision, char* buf, int buflen);
/* Same, for a plan created with `flags` (SHAFFT_SM100_PLAN_*). */
int shafft_sm100_plan_query_ex(int ndim, const int64_t* dims, int precision, int flags, char* buf,
                               int buflen);
int shafft_sm100_plan_query_axes(int ndim, const int64_t* dims, int precision, int flags, int naxes,
                                 const int* axes, char* buf, int buflen);

/* Run only step `step` (0 <= step < plan_launches()) of an execute with the
 * same buffer roles as shafft_sm100_execute.  Running steps 0..n-1 in order
 * on one stream is exactly one execute; used to time each kernel with
 * events placed between the launches. */
int shafft_sm100_execute_step(shafft_sm100_plan plan, int step, void* src, void* dst, int direction,
                              double scale, void* stream);

/* Algorithmic HBM bytes of step `step` (one compulsory read and write of
 * what the kernel touches), or 0 for an invalid step. */
int64_t shafft_sm100_step_bytes(shafft_sm100_plan plan, int step);

/* JSON description of a created plan: its steps in order, each pass with
 * its length, radices, tile width, buffers, row/column input and output,
 * tile count, shared memory, twiddle mode, kernel kind (fast, tc, bs, map)
 * and "prefetch", the L2 prefetch distance of the pass in quarter waves of
 * resident CTAs (0 = none; see SHAFFT_SM100_PREFETCH_ROW). */
int shafft_sm100_plan_describe(shafft_sm100_plan plan, char* buf, int buflen);

/* ---- Batched form: many independent transforms in one launch ----------
 * (no counterpart in the reference, which runs one plan per transform).
 *
 * count transforms; transform i has ndims[i] axes whose lengths follow in
 * `dims` (flattened, row-major, last axis fastest).  Every axis length must
 * factor into 2,3,5,7,11,13 and be <= 4096, or be <= 362 (direct DFT).
 * flags bit 0: autotune tile widths for lengths not yet in the tuning cache
 * (file SHAFFT_SM100_TUNE_CACHE, default ~/.cache/shafft_sm100_tune.txt).
 * execute: src[i] -> dst[i] for every i (device pointers; src[i] is only
 * read; src[i] == dst[i] is allowed), all transforms in one persistent kernel
 * launch replayed from a CUDA graph captured on the first call with that
 * direction and scale.  Asynchronous on `stream`. */
typedef struct shafft_sm100_batch_s* shafft_sm100_batch;
int shafft_sm100_batch_create(shafft_sm100_batch* out, int count, const int* ndims,
                              const int64_t* dims, int precision, int flags);
int shafft_sm100_batch_execute(shafft_sm100_batch b, void* const* src, void* const* dst,
                               int direction, double scale, void* stream);
int shafft_sm100_batch_destroy(shafft_sm100_batch b);
/* error flag of the last executes (call after synchronising) */
int shafft_sm100_batch_status(shafft_sm100_batch b);
/* Bound of each tile's wait for the previous pass of its transform: after
 * `polls` unsuccessful polls of the pass's completion counter (about 64 ns
 * apart) the tile sets the batch's error word and goes on, so the launch
 * always ends and shafft_sm100_batch_status then reports
 * SHAFFT_SM100_ECUDA.  0 restores the default (2^22 polls, far above any
 * legitimate wait).  A small bound exists to exercise that error path. */
int shafft_sm100_batch_set_wait_limit(shafft_sm100_batch b, unsigned polls);
/* algorithmic HBM bytes of one execute (read + write per pass) */
int64_t shafft_sm100_batch_bytes(shafft_sm100_batch b);
int shafft_sm100_batch_describe(shafft_sm100_batch b, char* buf, int buflen);

/* ---- Serving form: request loop with continuous admission ---------------
 * (no counterpart in the reference).  A server owns `streams` CUDA streams,
 * a dispatcher thread and a completion thread.  Requests (host input/output
 * buffers -- pinned for overlap) are admitted in arrival order as soon as
 * their two device buffers fit `budget_bytes` (resident plans count against
 * the budget; idle plans are evicted oldest first, and only when the
 * resident plans alone leave no room), issued on the stream with the
 * fewest bytes in flight (H2D, execute, D2H, in pieces of at most 8 MiB)
 * and so overlap with requests already running.  Requests with buffers of
 * 256 MiB or more copy one per direction at a time, fed to the copy engines
 * two pieces at a time and held back (at most 2 ms a piece) while smaller
 * requests' copies are pending, so a small request does not wait behind a
 * large transfer.  Requests of one shape share a plan instance when the plan
 * has no scratch.  The server's own memory pool is grown to the budget (or
 * to what the device can spare) at creation, so request buffers are carved
 * out of memory mapped up front.
 * wait() blocks until the request's output is in host_out and returns its
 * status and latency (submission to completion).  stats() reports completed
 * / failed counts, p50 / p99 / max latency, throughput, plan-instance
 * creations / evictions, the longest issue step and the p99 wait from
 * submission to issue as JSON.  Wait for every submitted request before
 * destroy. */
typedef struct shafft_sm100_server_s* shafft_sm100_server;
int shafft_sm100_server_create(shafft_sm100_server* out, size_t budget_bytes, int streams);
int shafft_sm100_server_submit(shafft_sm100_server s, int ndim, const int64_t* dims, int precision,
                               int direction, double scale, const void* host_in, void* host_out,
                               uint64_t* id);
int shafft_sm100_server_wait(shafft_sm100_server s, uint64_t id, double* latency_ms);
int shafft_sm100_server_stats(shafft_sm100_server s, char* buf, int buflen);
int shafft_sm100_server_reset_stats(shafft_sm100_server s);
int shafft_sm100_server_destroy(shafft_sm100_server s);

/* ---- Slab exchange helpers (distributed N-D transforms) -----------------
 * src / dst: device arrays, viewed as [outer][n][inner] row-major complex
 * elements (n = the axis being redistributed).  pack: dst = the nparts
 * blocks of that axis one after the other, block p = indices [start_p,
 * start_p + len_p) as an [outer][len_p][inner] array, (len_p, start_p) the
 * block partition of n (the first n % nparts blocks one element longer);
 * unpack is the inverse.  Asynchronous on `stream`.  Replaces the subarray
 * datatypes of the reference's MPI_Alltoallw exchange
 * (src/cpp/slab_nd.cpp:23-56). */
int shafft_sm100_pack_blocks(const void* src, void* dst, int64_t outer, int64_t n, int64_t inner,
                             int nparts, int precision, void* stream);
int shafft_sm100_unpack_blocks(const void* src, void* dst, int64_t outer, int64_t n, int64_t inner,
                               int nparts, int precision, void* stream);
/* data[k][c] *= exp(sign * 2*pi*i * ((col0 + c) * k mod N) / N) over a
 * rows x cols array (phase reduced in integers, FP64 sincospi): the twiddle
 * between the stages of the distributed four-step FFT1D (replaces the
 * reference's fft1dTwiddleKernel, 1d/fft1d_cooley_tukey_executor.hip:57-83). */
int shafft_sm100_twiddle_rows(void* data, int64_t rows, int64_t cols, int64_t col0, int64_t N,
                              int sign, int precision, void* stream);

/* Distributed Bluestein (FFT1D lengths not divisible by P^2; replaces the
 * reference's computeLocalChirpB / computeLocalConvolutionChirp,
 * 1d/fft1d_bluestein_executor.hip:150-198).  For i < count:
 *   b[i] = exp(-i*pi*n^2/N) at n = n0 + i < N, else 0
 *   v[i] = conj(b[m]) for m < N, conj(b[M-m]) for M-N < m < M, else 0, at
 *          m = m0 + i
 * (n^2 reduced mod 2N in integers, FP64 sincospi).  Either of b, v may be
 * NULL; M >= 2N - 1. */
int shafft_sm100_bluestein_chirps(void* b, void* v, int64_t N, int64_t M, int64_t n0, int64_t m0,
                                  int64_t count, int precision, void* stream);

/* dst[i] = conj_out(conj_in(src[i]) * factors[i] * scale) for i < valid and
 * 0 for valid <= i < count (src may equal dst): Bluestein's modulate,
 * spectrum-multiply and scale+demodulate steps (reference
 * 1d/fft1d_bluestein_executor.hip:38-129). */
int shafft_sm100_chirp_multiply(const void* src, void* dst, const void* factors, int64_t count,
                                int64_t valid, int conj_in, int conj_out, double scale, int precision,
                                void* stream);

/* ---- Real-to-complex / complex-to-real transforms ----------------------
 * (an extension: the reference supports C2C and Z2Z only,
 * docs/limitations.dox:51-60).  A real tensor dims[0..ndim) whose last length
 * L is even; its spectrum is the first L/2 + 1 frequencies of the last axis
 * (dims[0..ndim-1), L/2 + 1 complex elements, row-major), the rest following
 * by Hermitian symmetry -- the FFTW / cuFFT layout.  precision 0: float data
 * and complex64 spectrum; 1: double and complex128.
 *   execute_r2c: spectrum = scale * DFT(real)   (forward, exp(-2 pi i jk/n))
 *   execute_c2r: real = scale * unnormalised inverse DFT of the Hermitian
 *                spectrum, so c2r(r2c(x)) = N x for N = prod(dims)
 * Both read their input as scratch (its contents are undefined afterwards);
 * buffers are 16-byte aligned device memory, input and output distinct.
 * The plan owns a work array of prod(dims) / 2 complex elements (the
 * half-length complex view's transform) besides its C2C plan.  Asynchronous
 * on `stream`. */
typedef struct shafft_sm100_rplan_s* shafft_sm100_rplan;
int shafft_sm100_rplan_create(shafft_sm100_rplan* out, int ndim, const int64_t* dims, int precision);
int shafft_sm100_rplan_destroy(shafft_sm100_rplan plan);
/* complex elements of the spectrum: prod(dims[0..ndim-1)) * (L/2 + 1) */
int64_t shafft_sm100_rplan_spectrum_elements(shafft_sm100_rplan plan);
int shafft_sm100_execute_r2c(shafft_sm100_rplan plan, void* real_in, void* spec_out, double scale,
                             void* stream);
int shafft_sm100_execute_c2r(shafft_sm100_rplan plan, void* spec_in, void* real_out, double scale,
                             void* stream);

/* Device memory and stream helpers, so that callers above this ABI need no
 * CUDA runtime of their own (they replace the reference's allocBufferT /
 * freeBufferT / copyToBufferT / copyFromBufferT,
 * src/cpp/detail/buffer_utils.hpp:36-127, and its hipStreamSynchronize). */
#define SHAFFT_SM100_H2D 1
#define SHAFFT_SM100_D2H 2
#define SHAFFT_SM100_D2D 3
int shafft_sm100_malloc(void** ptr, size_t bytes);
int shafft_sm100_free(void* ptr);
/* stream == NULL: synchronous copy; otherwise asynchronous on that stream. */
int shafft_sm100_memcpy(void* dst, const void* src, size_t bytes, int kind, void* stream);
int shafft_sm100_stream_sync(void* stream);
/* Guard bytes (debugging aid, no counterpart in the reference): with
 * SHAFFT_SM100_CANARY=1 in the environment, shafft_sm100_malloc and the
 * plans' own table and scratch allocations put 256 bytes of a fixed pattern
 * before and after every block; shafft_sm100_free and plan destruction check
 * the guards of what they release, and this call checks every live block.
 * A changed guard byte (a kernel wrote outside its buffer) returns
 * SHAFFT_SM100_ECUDA with the buffer and offset in the message.  Reads the
 * guards with synchronous copies: call it with the device idle.  Returns 0
 * when the switch is off. */
int shafft_sm100_check_guards(void);

/* Name of the current CUDA device. */
int shafft_sm100_device_name(char* buf, int buflen);

/* Allocation-free 1-D C2C transform (no counterpart in the reference).
 *
 * For callers that cannot call cudaMalloc where they need the transform --
 * code running under an allocator lock, inside a framework callback that
 * forbids allocation, or within a fixed device-memory budget reserved up
 * front.  It takes only the caller's input and output device buffers of n
 * complex elements (in == out is allowed) and computes the unnormalised
 * length-n DFT (direction 0 forward, 1 backward) times `scale`, by
 * Bluestein's chirp-z method over a power-of-two convolution, for any n in
 * 1..2048.  Larger n is rejected with SHAFFT_SM100_EINVAL.
 *
 * All device state (chirp, kernel spectrum, twiddle and digit tables, two
 * convolution rows) lives in one file-scope __device__ array of about
 * 304 KiB that every device loading this library keeps until the process
 * exits.  Each call regenerates what it reads, so results do not depend on
 * earlier calls, but all calls on a device share the array: calls whose work
 * overlaps on the GPU race and corrupt each other -- issue them in order on
 * one stream.  The first call on each device does one-time set-up there:
 * it looks the array's address up with cudaGetSymbolAddress, and the first
 * call of each precision on that device raises the pass kernels' shared-
 * memory limit (cudaFuncSetAttribute).  Make one call of each precision you
 * use on every device before capturing a stream on it.
 * Asynchronous on `stream` (cudaStream_t, NULL = legacy default stream). */
int shafft_sm100_bluestein_noalloc(const void* in, void* out, int64_t n, int precision,
                                   int direction, double scale, void* stream);

/* Last CUDA runtime error code seen by this library on this thread. */
int shafft_sm100_last_cuda_error(void);

/* Human-readable message for the last error on this thread. */
const char* shafft_sm100_last_error_message(void);

/* Library version string. */
const char* shafft_sm100_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SHAFFT_SM100_H */
