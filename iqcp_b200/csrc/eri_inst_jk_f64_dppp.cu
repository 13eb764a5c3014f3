// Generated by gen_inst.py: jk f64 kernels for (dp|pp)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<double, 2, 1, 1, 1>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
