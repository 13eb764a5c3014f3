// Generated by gen_inst.py: jk f32 kernels for (dd|pp)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<float, 2, 2, 1, 1>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
