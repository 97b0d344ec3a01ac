/*
 * shafft.h -- C interface of SHAFFT, served by the B200 (sm_100a) backend.
 *
 * Every declaration below keeps the name, signature and meaning of the
 * reference's C API (include/shafft/shafft.h:42-845 of the SHAFFT project,
 * implemented in src/c/shafftc.cpp:60-555) so that existing C, C++ and
 * Fortran 2003 callers link unchanged.  Differences:
 *   - the GPU stream type is cudaStream_t (the reference's hipStream_t);
 *   - one extra entry point, shafftExecuteNormalized(), fuses an execute with
 *     the normalize() that follows it into the same HBM passes;
 *   - the backend is single-GPU: a communicator of one active rank.
 *
 * All functions return 0 (SHAFFT_SUCCESS) or a shafft_status_t code and never
 * throw; the last error of the calling thread is kept for the
 * shafftLastError*() queries.  Axis indices are 0-based, tensors row-major
 * with the last axis fastest.  After shafftExecute() the result lives in the
 * buffer that shafftGetBuffers() reports as `data` (data and work swap on
 * every execute).
 */
#ifndef SHAFFT_C_H
#define SHAFFT_C_H

#include <shafft/shafft_config.h>

#include <mpi.h>
#include <stddef.h>

#if SHAFFT_BACKEND_SM100
#include <cuda_runtime_api.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#if SHAFFT_BACKEND_SM100
/** Run the plan's kernels on `stream` (N-D or 1-D plan; after shafftPlan). */
int shafftSetStream(void* planPtr, cudaStream_t stream);
#endif

/** FFT precision: SHAFFT_C2C = complex<float>, SHAFFT_Z2Z = complex<double>. */
typedef enum { SHAFFT_C2C, SHAFFT_Z2Z } shafft_t;

/** Transform direction. */
typedef enum { SHAFFT_FORWARD, SHAFFT_BACKWARD } shafft_direction_t;

/** Layout selector for queries. */
typedef enum {
  SHAFFT_TENSOR_LAYOUT_CURRENT,
  SHAFFT_TENSOR_LAYOUT_INITIAL,
  SHAFFT_TENSOR_LAYOUT_REDISTRIBUTED
} shafft_tensor_layout_t;

/** Forward output-layout policy of N-D plans. */
typedef enum { SHAFFT_LAYOUT_REDISTRIBUTED = 0, SHAFFT_LAYOUT_INITIAL = 1 } shafft_transform_layout_t;

/** Status codes (same values as shafft::Status). */
typedef enum {
  SHAFFT_SUCCESS = 0,
  SHAFFT_ERR_NULLPTR = 1,
  SHAFFT_ERR_INVALID_COMM = 2,
  SHAFFT_ERR_NO_BUFFER = 3,
  SHAFFT_ERR_PLAN_NOT_INIT = 4,
  SHAFFT_ERR_INVALID_DIM = 5,
  SHAFFT_ERR_DIM_MISMATCH = 6,
  SHAFFT_ERR_INVALID_DECOMP = 7,
  SHAFFT_ERR_INVALID_FFTTYPE = 8,
  SHAFFT_ERR_ALLOC = 9,
  SHAFFT_ERR_BACKEND = 10,
  SHAFFT_ERR_MPI = 11,
  SHAFFT_ERR_INVALID_LAYOUT = 12,
  SHAFFT_ERR_SIZE_OVERFLOW = 13,
  SHAFFT_ERR_NOT_IMPL = 14,
  SHAFFT_ERR_INVALID_STATE = 15,
  SHAFFT_ERR_INTERNAL = 16
} shafft_status_t;

/** Subsystem an error came from.  In this backend SHAFFT_ERRSRC_HIP means
 *  the CUDA runtime and SHAFFT_ERRSRC_HIPFFT the sm_100a FFT kernel library
 *  (the enumerator names are kept for source compatibility). */
typedef enum {
  SHAFFT_ERRSRC_NONE = 0,
  SHAFFT_ERRSRC_MPI = 1,
  SHAFFT_ERRSRC_HIP = 2,
  SHAFFT_ERRSRC_HIPFFT = 3,
  SHAFFT_ERRSRC_FFTW = 4,
  SHAFFT_ERRSRC_SYSTEM = 5
} shafft_errsrc_t;

int shafftLastErrorStatus(void);
int shafftLastErrorSource(void);
int shafftLastErrorDomainCode(void);
/** Writes the message (NUL-terminated) and returns its length. */
int shafftLastErrorMessage(char* buf, int buflen);
void shafftClearLastError(void);
const char* shafftErrorSourceName(int source);

typedef enum { SHAFFT_MAXIMIZE_NDA, SHAFFT_MINIMIZE_NDA } shafft_decomposition_strategy_t;

typedef enum {
  SHAFFT_CONFIG_CHANGED_COMM_DIMS = (1 << 0),
  SHAFFT_CONFIG_CHANGED_NDA = (1 << 1),
  SHAFFT_CONFIG_INACTIVE_RANKS = (1 << 2),
  SHAFFT_CONFIG_RESOLVED = (1 << 3)
} shafft_config_flags_t;

/** Per-layout description of the local block (config-owned arrays). */
typedef struct shafft_nd_layout_t {
  size_t* subsize;
  size_t* offset;
  size_t localElements;
  int hasLocalElements;
  int* contiguousAxes;
  int* distributedAxes;
} shafft_nd_layout_t;

/** N-D configuration object; zero-initialise, then shafftConfigNDInit(). */
typedef struct shafft_nd_config_t {
  size_t structSize;
  int apiVersion;
  int ndim;
  shafft_t precision;
  size_t* globalShape;
  shafft_decomposition_strategy_t strategy;
  shafft_transform_layout_t outputPolicy;
  size_t memLimit;
  int* hintCommDims;
  int hintNda;
  int* commDims;
  int nda;
  int commSize;
  size_t allocElements;
  shafft_nd_layout_t initial;
  shafft_nd_layout_t output;
  int isActive;
  int activeRank;
  int activeSize;
  MPI_Comm worldComm;
  MPI_Comm activeComm;
  int nodeId;
  int nodeCount;
  char* hostname;
  size_t hostnameLen;
  char* deviceName;
  size_t deviceNameLen;
  int flags;
  int status;
  int reserved[8];
} shafft_nd_config_t;

typedef struct shafft_1d_layout_t {
  size_t localSize;
  size_t localStart;
  int hasLocalElements;
} shafft_1d_layout_t;

/** 1-D configuration object; zero-initialise, then shafftConfig1DInit(). */
typedef struct shafft_1d_config_t {
  size_t structSize;
  int apiVersion;
  size_t globalSize;
  shafft_t precision;
  shafft_1d_layout_t initial;
  shafft_1d_layout_t output;
  size_t allocElements;
  int isActive;
  int activeRank;
  int activeSize;
  MPI_Comm worldComm;
  MPI_Comm activeComm;
  int nodeId;
  int nodeCount;
  char* hostname;
  size_t hostnameLen;
  char* deviceName;
  size_t deviceNameLen;
  int flags;
  int status;
  int reserved[8];
} shafft_1d_config_t;

int shafftConfigNDInit(shafft_nd_config_t* cfg, int ndim, const size_t* globalShape,
                       shafft_t precision, const int* commDims, int hintNda,
                       shafft_decomposition_strategy_t strategy,
                       shafft_transform_layout_t outputPolicy, size_t memLimit, MPI_Comm comm);
void shafftConfigNDRelease(shafft_nd_config_t* cfg);
int shafftConfigNDResolve(shafft_nd_config_t* cfg);
int shafftNDInitFromConfig(void* planPtr, shafft_nd_config_t* cfg);
int shafftConfig1DInit(shafft_1d_config_t* cfg, size_t globalSize, shafft_t precision,
                       MPI_Comm comm);
void shafftConfig1DRelease(shafft_1d_config_t* cfg);
int shafftConfig1DResolve(shafft_1d_config_t* cfg);
int shafft1DInitFromConfig(void* planPtr, shafft_1d_config_t* cfg);
int shafftGetCommunicator(void* planPtr, MPI_Comm* outComm);

int shafftConfigurationND(int ndim, int* size, shafft_t precision, int* commDims, int* nda,
                          size_t* subsize, size_t* offset, int* commSize,
                          shafft_decomposition_strategy_t strategy, size_t memLimit,
                          MPI_Comm cComm);

int shafftNDCreate(void** outPlan);
int shafftNDInit(void* planPtr, int ndim, int commDims[], int dimensions[], shafft_t precision,
                 MPI_Comm cComm, shafft_transform_layout_t output_policy);
int shafftPlan(void* planPtr);
int shafftDestroy(void** planPtr);
int shafftGetLayout(void* planPtr, size_t* subsize, size_t* offset, shafft_tensor_layout_t layout);
int shafftGetAxes(void* planPtr, int* ca, int* da, shafft_tensor_layout_t layout);
int shafftGetAllocSize(void* plan, size_t* localAllocSize);
int shafftGetGlobalSize(void* plan, size_t* globalSize);
int shafftIsConfigured(void* plan, int* configured);
int shafftIsActive(void* plan, int* active);
int shafftSetBuffers(void* planPtr, void* data, void* work);
int shafftGetBuffers(void* planPtr, void** data, void** work);
int shafftExecute(void* planPtr, shafft_direction_t direction);
int shafftNormalize(void* planPtr);

/** Extension (no counterpart in the reference): identical result to
 *  shafftExecute(plan, direction) followed by shafftNormalize(plan), with the
 *  normalisation factor multiplied in by the last HBM pass of the transform
 *  instead of a separate read+write pass. */
int shafftExecuteNormalized(void* planPtr, shafft_direction_t direction);

int shafftConfiguration1D(size_t N, size_t* localN, size_t* localStart, size_t* localAllocSize,
                          shafft_t precision, MPI_Comm cComm);
int shafft1DCreate(void** outPlan);
int shafft1DInit(void* planPtr, size_t N, size_t localN, size_t localStart, shafft_t precision,
                 MPI_Comm cComm);

/** Device buffers (cudaMalloc) and host<->device copies. */
int shafftAllocBufferF(size_t count, void** buf);
int shafftAllocBufferD(size_t count, void** buf);
int shafftFreeBufferF(void* buf);
int shafftFreeBufferD(void* buf);
int shafftCopyToBufferF(void* dst, const void* src, size_t count);
int shafftCopyToBufferD(void* dst, const void* src, size_t count);
int shafftCopyFromBufferF(void* dst, const void* src, size_t count);
int shafftCopyFromBufferD(void* dst, const void* src, size_t count);

/** "sm100" (or the name the library was built to report). */
const char* shafftGetBackendName(void);
void shafftGetVersion(int* major, int* minor, int* patch);
const char* shafftGetVersionString(void);
int shafftFinalize(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SHAFFT_C_H */
