// Instantiation of the jk quartet kernels for bra class (dd|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_bra<2, 2>(int, const JKArgs&, cudaStream_t);
}  // namespace iqcp
