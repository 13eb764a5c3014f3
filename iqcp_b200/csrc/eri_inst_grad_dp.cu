// Instantiation of the grad quartet kernels for bra class (dp|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_bra<2, 1>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
