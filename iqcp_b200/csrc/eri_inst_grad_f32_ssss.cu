// Generated by gen_inst.py: grad f32 kernels for (ss|ss)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<float, 0, 0, 0, 0>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
