// Instantiation of the jk quartet kernels for bra class (pp|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_bra<1, 1>(int, const JKArgs&, cudaStream_t);
}  // namespace iqcp
