// Generated by gen_inst.py: store kernels for bra class (dp|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_store_bra<2, 1>(int, const StoreArgs&, cudaStream_t);
}  // namespace iqcp
