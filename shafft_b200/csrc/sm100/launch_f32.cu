// float (complex64) instantiation of the kernel launchers.
#include "launch_impl.cuh"
namespace shafft_sm100 {
template struct Launch<float>;
}
