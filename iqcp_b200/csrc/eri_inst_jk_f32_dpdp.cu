// Generated by gen_inst.py: jk f32 kernels for (dp|dp)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<float, 2, 1, 2, 1>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
