/* Entry points of SHAFFT's Fortran 2003 binding.
 *
 * The reference's Fortran module (src/f03/shafft.f03:198-663) binds, besides
 * the public C ABI of shafft.h, to the C functions below: wrappers taking
 * Fortran MPI handles (MPI_Fint) and the accessors its derived types use to
 * copy the configuration objects field by field (src/f03/shafftf03.h:1-200,
 * src/f03/shafftf03.cpp:11-344).  libshafft.so exports every one of them, so
 * that module compiles and links against this library unchanged.
 *
 * Accessors of a NULL config return 0 (MPI_COMM_NULL's handle for the
 * communicators) and copy nothing; array getters copy ndim entries into a
 * caller buffer; string getters copy at most maxLen bytes and terminate the
 * copy with NUL when it is shorter than maxLen. */
#ifndef SHAFFT_F03_H
#define SHAFFT_F03_H

#include <mpi.h>
#include <shafft/shafft.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* wrappers taking a Fortran communicator handle */
int shafftConfigurationNDf03(int ndim, int* size, shafft_t precision, int* commDims, int* nda,
                             size_t* subsize, size_t* offset, int* commSize,
                             shafft_decomposition_strategy_t strategy, size_t memLimit,
                             MPI_Fint* fHandle);
int shafftNDInitf03(void* planPtr, int ndim, int commDims[], int dimensions[], shafft_t precision,
                    MPI_Fint* fHandle, shafft_transform_layout_t* outputPolicy);
int shafftConfiguration1Df03(size_t N, size_t* localN, size_t* localStart, size_t* localAllocSize,
                             shafft_t precision, MPI_Fint* fHandle);
int shafft1DInitf03(void* planPtr, size_t N, size_t localN, size_t localStart, shafft_t precision,
                    MPI_Fint* fHandle);
int shafftGetCommunicatorf03(void* planPtr, MPI_Fint* outFint);

/* configuration objects on the C heap (zero-initialised) */
shafft_nd_config_t* shafftConfigNDAllocf03(void);
void shafftConfigNDFreef03(shafft_nd_config_t* cfg);
shafft_1d_config_t* shafftConfig1DAllocf03(void);
void shafftConfig1DFreef03(shafft_1d_config_t* cfg);
int shafftConfigNDInitf03(shafft_nd_config_t* cfg, int ndim, const size_t* globalShape,
                          shafft_t precision, const int* commDims, int hintNda,
                          shafft_decomposition_strategy_t strategy,
                          shafft_transform_layout_t outputPolicy, size_t memLimit, MPI_Fint* fComm);
int shafftConfigNDResolvef03(shafft_nd_config_t* cfg);
int shafftNDInitFromConfigf03(void* planPtr, shafft_nd_config_t* cfg);
int shafftConfig1DInitf03(shafft_1d_config_t* cfg, size_t globalSize, shafft_t precision,
                          MPI_Fint* fComm);
int shafftConfig1DResolvef03(shafft_1d_config_t* cfg);
int shafft1DInitFromConfigf03(void* planPtr, shafft_1d_config_t* cfg);

/* N-D accessors */
int shafftConfigNDGetNdim(const shafft_nd_config_t* cfg);
int shafftConfigNDGetPrecision(const shafft_nd_config_t* cfg);
size_t shafftConfigNDGetAllocElements(const shafft_nd_config_t* cfg);
int shafftConfigNDGetIsActive(const shafft_nd_config_t* cfg);
int shafftConfigNDGetActiveRank(const shafft_nd_config_t* cfg);
int shafftConfigNDGetActiveSize(const shafft_nd_config_t* cfg);
int shafftConfigNDGetNda(const shafft_nd_config_t* cfg);
int shafftConfigNDGetCommSize(const shafft_nd_config_t* cfg);
int shafftConfigNDGetStatus(const shafft_nd_config_t* cfg);
int shafftConfigNDGetOutputPolicy(const shafft_nd_config_t* cfg);
int shafftConfigNDGetStrategy(const shafft_nd_config_t* cfg);
size_t shafftConfigNDGetMemLimit(const shafft_nd_config_t* cfg);
int shafftConfigNDGetHintNda(const shafft_nd_config_t* cfg);
int shafftConfigNDGetFlags(const shafft_nd_config_t* cfg);
MPI_Fint shafftConfigNDGetWorldComm(const shafft_nd_config_t* cfg);
MPI_Fint shafftConfigNDGetActiveComm(const shafft_nd_config_t* cfg);
int shafftConfigNDGetNodeId(const shafft_nd_config_t* cfg);
int shafftConfigNDGetNodeCount(const shafft_nd_config_t* cfg);
size_t shafftConfigNDGetHostnameLen(const shafft_nd_config_t* cfg);
void shafftConfigNDGetHostname(const shafft_nd_config_t* cfg, char* out, size_t maxLen);
size_t shafftConfigNDGetDeviceNameLen(const shafft_nd_config_t* cfg);
void shafftConfigNDGetDeviceName(const shafft_nd_config_t* cfg, char* out, size_t maxLen);
void shafftConfigNDGetGlobalShape(const shafft_nd_config_t* cfg, size_t* out);
void shafftConfigNDGetCommDims(const shafft_nd_config_t* cfg, int* out);
void shafftConfigNDGetHintCommDims(const shafft_nd_config_t* cfg, int* out);
void shafftConfigNDGetInitialSubsize(const shafft_nd_config_t* cfg, size_t* out);
void shafftConfigNDGetInitialOffset(const shafft_nd_config_t* cfg, size_t* out);
void shafftConfigNDGetOutputSubsize(const shafft_nd_config_t* cfg, size_t* out);
void shafftConfigNDGetOutputOffset(const shafft_nd_config_t* cfg, size_t* out);
void shafftConfigNDSetOutputPolicy(shafft_nd_config_t* cfg, int pol);
void shafftConfigNDSetStrategy(shafft_nd_config_t* cfg, int s);
void shafftConfigNDSetMemLimit(shafft_nd_config_t* cfg, size_t limit);
void shafftConfigNDSetHintNda(shafft_nd_config_t* cfg, int nda);
void shafftConfigNDSetHintCommDims(shafft_nd_config_t* cfg, const int* dims);

/* 1-D accessors */
size_t shafftConfig1DGetGlobalSize(const shafft_1d_config_t* cfg);
int shafftConfig1DGetPrecision(const shafft_1d_config_t* cfg);
size_t shafftConfig1DGetAllocElements(const shafft_1d_config_t* cfg);
int shafftConfig1DGetIsActive(const shafft_1d_config_t* cfg);
int shafftConfig1DGetActiveRank(const shafft_1d_config_t* cfg);
int shafftConfig1DGetActiveSize(const shafft_1d_config_t* cfg);
int shafftConfig1DGetStatus(const shafft_1d_config_t* cfg);
int shafftConfig1DGetFlags(const shafft_1d_config_t* cfg);
MPI_Fint shafftConfig1DGetWorldComm(const shafft_1d_config_t* cfg);
MPI_Fint shafftConfig1DGetActiveComm(const shafft_1d_config_t* cfg);
int shafftConfig1DGetNodeId(const shafft_1d_config_t* cfg);
int shafftConfig1DGetNodeCount(const shafft_1d_config_t* cfg);
size_t shafftConfig1DGetHostnameLen(const shafft_1d_config_t* cfg);
void shafftConfig1DGetHostname(const shafft_1d_config_t* cfg, char* out, size_t maxLen);
size_t shafftConfig1DGetDeviceNameLen(const shafft_1d_config_t* cfg);
void shafftConfig1DGetDeviceName(const shafft_1d_config_t* cfg, char* out, size_t maxLen);
size_t shafftConfig1DGetInitialLocalSize(const shafft_1d_config_t* cfg);
size_t shafftConfig1DGetInitialLocalStart(const shafft_1d_config_t* cfg);
size_t shafftConfig1DGetOutputLocalSize(const shafft_1d_config_t* cfg);
size_t shafftConfig1DGetOutputLocalStart(const shafft_1d_config_t* cfg);

#ifdef __cplusplus
}
#endif

#endif /* SHAFFT_F03_H */
