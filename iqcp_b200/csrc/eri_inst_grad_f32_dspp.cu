// Generated by gen_inst.py: grad f32 kernels for (ds|pp)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<float, 2, 0, 1, 1>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
