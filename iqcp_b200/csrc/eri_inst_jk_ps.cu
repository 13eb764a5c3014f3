// Instantiation of the jk quartet kernels for bra class (ps|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_bra<1, 0>(int, const JKArgs&, cudaStream_t);
}  // namespace iqcp
