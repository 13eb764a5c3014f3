// Generated by gen_inst.py: jk dispatch for bra class (ss|
#include "eri_launch.cuh"

namespace iqcp {
extern template cudaError_t launch_jk_variant<double, 0, 0, 0, 0>(const JKArgs&, cudaStream_t);
extern template cudaError_t launch_jk_variant<float, 0, 0, 0, 0>(const JKArgs&, cudaStream_t);
template cudaError_t launch_jk_bra<0, 0>(int, const JKArgs&, cudaStream_t);
}  // namespace iqcp
