// Generated by gen_inst.py: jk f64 kernels for (dd|dp)
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_jk_variant<double, 2, 2, 2, 1>(const JKArgs&, cudaStream_t);
}  // namespace iqcp
