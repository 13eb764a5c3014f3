// Generated by gen_inst.py: grad f64 kernels for (ds|ss)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_grad_variant<double, 2, 0, 0, 0>(const GradArgs&, cudaStream_t);
}  // namespace iqcp
