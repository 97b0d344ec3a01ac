/* shafft_config.h -- build configuration of the B200 (sm_100a) SHAFFT backend.
 * Mirrors the fields of the reference's generated header
 * (cmake/shafft_config.h.in:1-21); this build has exactly one backend. */
#ifndef SHAFFT_CONFIG_H
#define SHAFFT_CONFIG_H

#define SHAFFT_BACKEND_HIPFFT 0
#define SHAFFT_BACKEND_FFTW 0
/* GPU backend: hand-written sm_100a CUDA kernels (libshafft_sm100.so). */
#define SHAFFT_BACKEND_SM100 1

#ifndef SHAFFT_BACKEND_NAME
#define SHAFFT_BACKEND_NAME "sm100"
#endif

/* Single GPU, single rank: no device pointers are ever handed to MPI. */
#define SHAFFT_GPU_AWARE_MPI 0

#define SHAFFT_VERSION_MAJOR 1
#define SHAFFT_VERSION_MINOR 1
#define SHAFFT_VERSION_PATCH 0
#define SHAFFT_VERSION_SUFFIX "-alpha"

#define SHAFFT_STRINGIFY_IMPL(x) #x
#define SHAFFT_STRINGIFY(x) SHAFFT_STRINGIFY_IMPL(x)

#endif /* SHAFFT_CONFIG_H */
