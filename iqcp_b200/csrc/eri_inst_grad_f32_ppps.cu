// Generated by gen_inst.py: grad f32 kernels for (pp|ps)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<float, 1, 1, 1, 0>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
