// double (complex128) instantiation of the kernel launchers.
#define SHAFFT_INSTANTIATE_F64 1
#include "launch_impl.cuh"
namespace shafft_sm100 {
template struct Launch<double>;
}
