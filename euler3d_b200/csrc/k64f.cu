// FP64 batch kernels built with fused multiply-add contraction (see the
// Makefile).  They run the FP64 finishing phase of batched solves: the same
// discrete equations as the bit-identical path, converging to the same
// solution, with results that differ from it in the last bits.  First-order
// AUSM forms each cell's side quantities once (E3D_SHARED_SIDES, kernels.cuh).
#define E3D_BATCH_NS batch_fast
#define E3D_SHARED_SIDES
#include "batch_launch.cuh"

namespace e3d {

template int batch_fast::persistent_blocks_per_sm<double>(int, int, int, bool);
template cudaError_t batch_fast::launch_persistent<double>(const FusedView<double>&, const FusedView<double>&,
                                                           const Physics&, const PersistArgs&, int, int, int, bool, int,
                                                           cudaStream_t);
template cudaError_t batch_fast::launch_tiled_iterations<double>(const FusedView<double>&, const FusedView<double>&,
                                                                 const Physics&, const PersistArgs&, int, int, int, bool,
                                                                 cudaStream_t);

}  // namespace e3d
