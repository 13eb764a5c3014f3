// Generated by gen_inst.py: grad f64 kernels for (dd|pp)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<double, 2, 2, 1, 1>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
