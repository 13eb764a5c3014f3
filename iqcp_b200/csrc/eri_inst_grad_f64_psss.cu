// Generated by gen_inst.py: grad f64 kernels for (ps|ss)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<double, 1, 0, 0, 0>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
