// Generated by gen_inst.py: jk f64 kernels for (pp|ss)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<double, 1, 1, 0, 0>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
