// Generated by gen_inst.py: jk dispatch for bra class (ds|
#include "eri_launch.cuh"

namespace iqcp {
extern template cudaError_t launch_jk_variant<double, 2, 0, 0, 0>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<double, 2, 0, 1, 0>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<double, 2, 0, 1, 1>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<double, 2, 0, 2, 0>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<float, 2, 0, 0, 0>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<float, 2, 0, 1, 0>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<float, 2, 0, 1, 1>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<float, 2, 0, 2, 0>(const JKArgs&, cudaStream_t);
template cudaError_t launch_jk_bra<2, 0>(int, const JKArgs&, cudaStream_t);
}  // namespace iqcp
