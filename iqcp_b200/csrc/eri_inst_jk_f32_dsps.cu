// Generated by gen_inst.py: jk f32 kernels for (ds|ps)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<float, 2, 0, 1, 0>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
