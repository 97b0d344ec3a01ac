// Enumerations of the SHAFFT C++ API (same enumerators and order as the
// reference's include/shafft/shafft_enums.hpp:18-48).
#ifndef SHAFFT_ENUMS_HPP
#define SHAFFT_ENUMS_HPP

namespace shafft {

/// Transform direction: FORWARD uses exp(-2*pi*i*jk/n), BACKWARD exp(+...).
enum class FFTDirection { FORWARD, BACKWARD };

/// Element precision: C2C = complex<float>, Z2Z = complex<double>.
enum class FFTType { C2C, Z2Z };

/// Which layout a query refers to.
enum class TensorLayout { CURRENT, INITIAL, REDISTRIBUTED };

}  // namespace shafft

#endif  // SHAFFT_ENUMS_HPP
