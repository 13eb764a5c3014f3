// Generated by gen_inst.py: jk f64 kernels for (ss|ss)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<double, 0, 0, 0, 0>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
