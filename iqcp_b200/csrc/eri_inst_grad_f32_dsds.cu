// Generated by gen_inst.py: grad f32 kernels for (ds|ds)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<float, 2, 0, 2, 0>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
