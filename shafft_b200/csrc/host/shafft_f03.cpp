// Fortran-binding entry points of libshafft.so (declared in
// include/shafft/shafft_f03.h): the handle-converting wrappers and the
// configuration-object accessors that SHAFFT's Fortran 2003 module binds to
// (reference interface: src/f03/shafftf03.h, src/f03/shafftf03.cpp:11-344).
// Everything here is host bookkeeping over the public C ABI; no device work.
#include <shafft/shafft_f03.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace {

template <typename T>
void copy_n(const T* src, int n, T* out) {
  if (src && out && n > 0) std::memcpy(out, src, sizeof(T) * (size_t)n);
}

void copy_text(const char* src, size_t len, char* out, size_t maxLen) {
  if (!out || maxLen == 0) return;
  const size_t n = src ? std::min(len, maxLen) : 0;
  if (n) std::memcpy(out, src, n);
  if (n < maxLen) out[n] = '\0';
}

MPI_Comm from_fortran(const MPI_Fint* h) { return h ? MPI_Comm_f2c(*h) : MPI_COMM_NULL; }

}  // namespace

extern "C" {

// ---- wrappers taking Fortran communicator handles ----

int shafftConfigurationNDf03(int ndim, int* size, shafft_t precision, int* commDims, int* nda,
                             size_t* subsize, size_t* offset, int* commSize,
                             shafft_decomposition_strategy_t strategy, size_t memLimit,
                             MPI_Fint* fHandle) {
  if (!fHandle) return SHAFFT_ERR_NULLPTR;
  return shafftConfigurationND(ndim, size, precision, commDims, nda, subsize, offset, commSize,
                               strategy, memLimit, from_fortran(fHandle));
}

int shafftNDInitf03(void* planPtr, int ndim, int commDims[], int dimensions[], shafft_t precision,
                    MPI_Fint* fHandle, shafft_transform_layout_t* outputPolicy) {
  if (!fHandle || !outputPolicy) return SHAFFT_ERR_NULLPTR;
  return shafftNDInit(planPtr, ndim, commDims, dimensions, precision, from_fortran(fHandle),
                      *outputPolicy);
}

int shafftConfiguration1Df03(size_t N, size_t* localN, size_t* localStart, size_t* localAllocSize,
                             shafft_t precision, MPI_Fint* fHandle) {
  if (!fHandle) return SHAFFT_ERR_NULLPTR;
  return shafftConfiguration1D(N, localN, localStart, localAllocSize, precision,
                               from_fortran(fHandle));
}

int shafft1DInitf03(void* planPtr, size_t N, size_t localN, size_t localStart, shafft_t precision,
                    MPI_Fint* fHandle) {
  if (!fHandle) return SHAFFT_ERR_NULLPTR;
  return shafft1DInit(planPtr, N, localN, localStart, precision, from_fortran(fHandle));
}

int shafftGetCommunicatorf03(void* planPtr, MPI_Fint* outFint) {
  if (!outFint) return SHAFFT_ERR_NULLPTR;
  MPI_Comm c = MPI_COMM_NULL;
  const int rc = shafftGetCommunicator(planPtr, &c);
  if (rc == 0) *outFint = MPI_Comm_c2f(c);
  return rc;
}

// ---- configuration objects ----

shafft_nd_config_t* shafftConfigNDAllocf03(void) {
  return static_cast<shafft_nd_config_t*>(std::calloc(1, sizeof(shafft_nd_config_t)));
}
void shafftConfigNDFreef03(shafft_nd_config_t* cfg) { std::free(cfg); }
shafft_1d_config_t* shafftConfig1DAllocf03(void) {
  return static_cast<shafft_1d_config_t*>(std::calloc(1, sizeof(shafft_1d_config_t)));
}
void shafftConfig1DFreef03(shafft_1d_config_t* cfg) { std::free(cfg); }

int shafftConfigNDInitf03(shafft_nd_config_t* cfg, int ndim, const size_t* globalShape,
                          shafft_t precision, const int* commDims, int hintNda,
                          shafft_decomposition_strategy_t strategy,
                          shafft_transform_layout_t outputPolicy, size_t memLimit, MPI_Fint* fComm) {
  if (!fComm) return SHAFFT_ERR_NULLPTR;
  return shafftConfigNDInit(cfg, ndim, globalShape, precision, commDims, hintNda, strategy,
                            outputPolicy, memLimit, from_fortran(fComm));
}
int shafftConfigNDResolvef03(shafft_nd_config_t* cfg) { return shafftConfigNDResolve(cfg); }
int shafftNDInitFromConfigf03(void* planPtr, shafft_nd_config_t* cfg) {
  return shafftNDInitFromConfig(planPtr, cfg);
}
int shafftConfig1DInitf03(shafft_1d_config_t* cfg, size_t globalSize, shafft_t precision,
                          MPI_Fint* fComm) {
  if (!fComm) return SHAFFT_ERR_NULLPTR;
  return shafftConfig1DInit(cfg, globalSize, precision, from_fortran(fComm));
}
int shafftConfig1DResolvef03(shafft_1d_config_t* cfg) { return shafftConfig1DResolve(cfg); }
int shafft1DInitFromConfigf03(void* planPtr, shafft_1d_config_t* cfg) {
  return shafft1DInitFromConfig(planPtr, cfg);
}

// ---- N-D accessors ----

#define SHAFFT_ND_GET(NAME, TYPE, EXPR) \
  TYPE shafftConfigND##NAME(const shafft_nd_config_t* cfg) { return cfg ? (TYPE)(EXPR) : (TYPE)0; }
SHAFFT_ND_GET(GetNdim, int, cfg->ndim)
SHAFFT_ND_GET(GetPrecision, int, cfg->precision)
SHAFFT_ND_GET(GetAllocElements, size_t, cfg->allocElements)
SHAFFT_ND_GET(GetIsActive, int, cfg->isActive)
SHAFFT_ND_GET(GetActiveRank, int, cfg->activeRank)
SHAFFT_ND_GET(GetActiveSize, int, cfg->activeSize)
SHAFFT_ND_GET(GetNda, int, cfg->nda)
SHAFFT_ND_GET(GetCommSize, int, cfg->commSize)
SHAFFT_ND_GET(GetStatus, int, cfg->status)
SHAFFT_ND_GET(GetOutputPolicy, int, cfg->outputPolicy)
SHAFFT_ND_GET(GetStrategy, int, cfg->strategy)
SHAFFT_ND_GET(GetMemLimit, size_t, cfg->memLimit)
SHAFFT_ND_GET(GetHintNda, int, cfg->hintNda)
SHAFFT_ND_GET(GetFlags, int, cfg->flags)
SHAFFT_ND_GET(GetNodeId, int, cfg->nodeId)
SHAFFT_ND_GET(GetNodeCount, int, cfg->nodeCount)
SHAFFT_ND_GET(GetHostnameLen, size_t, cfg->hostnameLen)
SHAFFT_ND_GET(GetDeviceNameLen, size_t, cfg->deviceNameLen)
#undef SHAFFT_ND_GET

MPI_Fint shafftConfigNDGetWorldComm(const shafft_nd_config_t* cfg) {
  return MPI_Comm_c2f(cfg ? cfg->worldComm : MPI_COMM_NULL);
}
MPI_Fint shafftConfigNDGetActiveComm(const shafft_nd_config_t* cfg) {
  return MPI_Comm_c2f(cfg ? cfg->activeComm : MPI_COMM_NULL);
}
void shafftConfigNDGetHostname(const shafft_nd_config_t* cfg, char* out, size_t maxLen) {
  if (cfg) copy_text(cfg->hostname, cfg->hostnameLen, out, maxLen);
}
void shafftConfigNDGetDeviceName(const shafft_nd_config_t* cfg, char* out, size_t maxLen) {
  if (cfg) copy_text(cfg->deviceName, cfg->deviceNameLen, out, maxLen);
}
void shafftConfigNDGetGlobalShape(const shafft_nd_config_t* cfg, size_t* out) {
  if (cfg) copy_n(cfg->globalShape, cfg->ndim, out);
}
void shafftConfigNDGetCommDims(const shafft_nd_config_t* cfg, int* out) {
  if (cfg) copy_n(cfg->commDims, cfg->ndim, out);
}
void shafftConfigNDGetHintCommDims(const shafft_nd_config_t* cfg, int* out) {
  if (cfg) copy_n(cfg->hintCommDims, cfg->ndim, out);
}
void shafftConfigNDGetInitialSubsize(const shafft_nd_config_t* cfg, size_t* out) {
  if (cfg) copy_n(cfg->initial.subsize, cfg->ndim, out);
}
void shafftConfigNDGetInitialOffset(const shafft_nd_config_t* cfg, size_t* out) {
  if (cfg) copy_n(cfg->initial.offset, cfg->ndim, out);
}
void shafftConfigNDGetOutputSubsize(const shafft_nd_config_t* cfg, size_t* out) {
  if (cfg) copy_n(cfg->output.subsize, cfg->ndim, out);
}
void shafftConfigNDGetOutputOffset(const shafft_nd_config_t* cfg, size_t* out) {
  if (cfg) copy_n(cfg->output.offset, cfg->ndim, out);
}

// setters of the fields a Fortran caller may change before re-resolving
void shafftConfigNDSetOutputPolicy(shafft_nd_config_t* cfg, int pol) {
  if (cfg) cfg->outputPolicy = (shafft_transform_layout_t)pol;
}
void shafftConfigNDSetStrategy(shafft_nd_config_t* cfg, int s) {
  if (cfg) cfg->strategy = (shafft_decomposition_strategy_t)s;
}
void shafftConfigNDSetMemLimit(shafft_nd_config_t* cfg, size_t limit) {
  if (cfg) cfg->memLimit = limit;
}
void shafftConfigNDSetHintNda(shafft_nd_config_t* cfg, int nda) {
  if (cfg) cfg->hintNda = nda;
}
void shafftConfigNDSetHintCommDims(shafft_nd_config_t* cfg, const int* dims) {
  // the hint array belongs to the config (allocated by shafftConfigNDInit)
  if (cfg) copy_n(dims, cfg->hintCommDims ? cfg->ndim : 0, cfg->hintCommDims);
}

// ---- 1-D accessors ----

#define SHAFFT_1D_GET(NAME, TYPE, EXPR) \
  TYPE shafftConfig1D##NAME(const shafft_1d_config_t* cfg) { return cfg ? (TYPE)(EXPR) : (TYPE)0; }
SHAFFT_1D_GET(GetGlobalSize, size_t, cfg->globalSize)
SHAFFT_1D_GET(GetPrecision, int, cfg->precision)
SHAFFT_1D_GET(GetAllocElements, size_t, cfg->allocElements)
SHAFFT_1D_GET(GetIsActive, int, cfg->isActive)
SHAFFT_1D_GET(GetActiveRank, int, cfg->activeRank)
SHAFFT_1D_GET(GetActiveSize, int, cfg->activeSize)
SHAFFT_1D_GET(GetStatus, int, cfg->status)
SHAFFT_1D_GET(GetFlags, int, cfg->flags)
SHAFFT_1D_GET(GetNodeId, int, cfg->nodeId)
SHAFFT_1D_GET(GetNodeCount, int, cfg->nodeCount)
SHAFFT_1D_GET(GetHostnameLen, size_t, cfg->hostnameLen)
SHAFFT_1D_GET(GetDeviceNameLen, size_t, cfg->deviceNameLen)
SHAFFT_1D_GET(GetInitialLocalSize, size_t, cfg->initial.localSize)
SHAFFT_1D_GET(GetInitialLocalStart, size_t, cfg->initial.localStart)
SHAFFT_1D_GET(GetOutputLocalSize, size_t, cfg->output.localSize)
SHAFFT_1D_GET(GetOutputLocalStart, size_t, cfg->output.localStart)
#undef SHAFFT_1D_GET

MPI_Fint shafftConfig1DGetWorldComm(const shafft_1d_config_t* cfg) {
  return MPI_Comm_c2f(cfg ? cfg->worldComm : MPI_COMM_NULL);
}
MPI_Fint shafftConfig1DGetActiveComm(const shafft_1d_config_t* cfg) {
  return MPI_Comm_c2f(cfg ? cfg->activeComm : MPI_COMM_NULL);
}
void shafftConfig1DGetHostname(const shafft_1d_config_t* cfg, char* out, size_t maxLen) {
  if (cfg) copy_text(cfg->hostname, cfg->hostnameLen, out, maxLen);
}
void shafftConfig1DGetDeviceName(const shafft_1d_config_t* cfg, char* out, size_t maxLen) {
  if (cfg) copy_text(cfg->deviceName, cfg->deviceNameLen, out, maxLen);
}

}  // extern "C"
