// Generated by gen_inst.py: grad dispatch for bra class (dp|
#include "eri_launch.cuh"

namespace iqcp {
extern template cudaError_t launch_grad_variant<double, 2, 1, 0, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<double, 2, 1, 1, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<double, 2, 1, 1, 1>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<double, 2, 1, 2, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<double, 2, 1, 2, 1>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 2, 1, 0, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 2, 1, 1, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 2, 1, 1, 1>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 2, 1, 2, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 2, 1, 2, 1>(const GradArgs&, cudaStream_t);
template cudaError_t launch_grad_bra<2, 1>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
