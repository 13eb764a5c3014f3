// Instantiation of the grad quartet kernels for bra class (ss|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_bra<0, 0>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
