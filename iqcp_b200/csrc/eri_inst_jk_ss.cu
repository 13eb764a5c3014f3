// Instantiation of the jk quartet kernels for bra class (ss|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_bra<0, 0>(int, const JKArgs&, cudaStream_t);
}  // namespace iqcp
