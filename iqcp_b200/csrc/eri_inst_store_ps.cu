// Generated by gen_inst.py: store kernels for bra class (ps|
#include "eri_launch.cuh"

namespace iqcp {
template cudaError_t launch_store_bra<1, 0>(int, const StoreArgs&, cudaStream_t);
}  // namespace iqcp
