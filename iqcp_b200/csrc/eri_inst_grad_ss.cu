// Generated by gen_inst.py: grad dispatch for bra class (ss|
#include "eri_launch.cuh"

namespace iqcp {
extern template cudaError_t launch_grad_variant<double, 0, 0, 0, 0>(const GradArgs&, cudaStream_t);
extern template cudaError_t launch_grad_variant<float, 0, 0, 0, 0>(const GradArgs&, cudaStream_t);
template cudaError_t launch_grad_bra<0, 0>(int, const GradArgs&, cudaStream_t);
}  // namespace iqcp
