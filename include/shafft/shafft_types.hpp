// Core types of the SHAFFT C++ API (values and names as in the reference's
// include/shafft/shafft_types.hpp:71-160).
#ifndef SHAFFT_TYPES_H
#define SHAFFT_TYPES_H

#include <shafft/shafft_config.h>
#include <shafft/shafft_enums.hpp>

#include <complex>
#include <cstddef>
#include <cstdint>
#include <mpi.h>
#include <vector>

namespace shafft {

/// Compute backends a SHAFFT build can carry; this build is SM100.
enum class Backend { HIPFFT, FFTW, SM100 };

constexpr Backend backend() noexcept { return Backend::SM100; }
constexpr const char* backendName() noexcept { return SHAFFT_BACKEND_NAME; }

using complexf = std::complex<float>;
using complexd = std::complex<double>;

/// Plan lifecycle: init() -> CONFIGURED, plan() -> PLANNED.
enum class PlanState { UNINITIALIZED, CONFIGURED, PLANNED };

/// Status codes returned by every entry point (0 = success).
enum class Status : int {
  SUCCESS = 0,
  ERR_NULLPTR = 1,
  ERR_INVALID_COMM = 2,
  ERR_NO_BUFFER = 3,
  ERR_PLAN_NOT_INIT = 4,
  ERR_INVALID_DIM = 5,
  ERR_DIM_MISMATCH = 6,
  ERR_INVALID_DECOMP = 7,
  ERR_INVALID_FFTTYPE = 8,
  ERR_ALLOC = 9,
  ERR_BACKEND = 10,
  ERR_MPI = 11,
  ERR_INVALID_LAYOUT = 12,
  ERR_SIZE_OVERFLOW = 13,
  ERR_NOT_IMPL = 14,
  ERR_INVALID_STATE = 15,
  ERR_INTERNAL = 16
};

enum class DecompositionStrategy { MAXIMIZE_NDA, MINIMIZE_NDA };

enum class PlanType { PLAN_ND, PLAN_1D };

/// Forward-output layout policy (only observable with >1 rank).
enum class TransformLayout { REDISTRIBUTED, INITIAL };

enum class ConfigPolicy { AUTO_ADJUST = 0, EXACT = 1 };

/// Product of the first ndim entries of array, accumulated in U.
template <typename T, typename U>
U product(T* array, int ndim) {
  U prod = static_cast<U>(1);
  for (int i = 0; i < ndim; i++) prod *= static_cast<U>(array[i]);
  return prod;
}

}  // namespace shafft

#endif  // SHAFFT_TYPES_H
