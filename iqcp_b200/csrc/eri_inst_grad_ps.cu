// Instantiation of the grad quartet kernels for bra class (ps|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_bra<1, 0>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
