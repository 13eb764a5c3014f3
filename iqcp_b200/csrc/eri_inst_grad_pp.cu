// Generated by gen_inst.py: grad dispatch for bra class (pp|
#include "eri_launch.cuh"

namespace iqcp {
extern template cudaError_t launch_grad_variant<double, 1, 1, 0, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<double, 1, 1, 1, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<double, 1, 1, 1, 1>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 1, 1, 0, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 1, 1, 1, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 1, 1, 1, 1>(const GradArgs&, cudaStream_t);
template cudaError_t launch_grad_bra<1, 1>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
