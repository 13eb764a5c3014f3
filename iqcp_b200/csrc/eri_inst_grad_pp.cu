// Instantiation of the grad quartet kernels for bra class (pp|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_bra<1, 1>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
