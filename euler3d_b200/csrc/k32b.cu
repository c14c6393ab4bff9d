// FP32 batch kernels (persistent and tiled per-pass forms), built with the
// FP32 variant's flags.  Batches are checked against the single-case FP32 path
// within the FP32 variant's tolerance, not bit for bit, so first-order AUSM
// here forms each cell's side quantities once (E3D_SHARED_SIDES, kernels.cuh);
// the single-case FP32 path (k32.cu) keeps the reference's operation order.
#define E3D_SHARED_SIDES
#include "batch_launch.cuh"

namespace e3d {

template int batch::persistent_blocks_per_sm<float>(int, int, int, bool);
template cudaError_t batch::launch_persistent<float>(const FusedView<float>&, const FusedView<float>&, const Physics&,
                                                     const PersistArgs&, int, int, int, bool, int, cudaStream_t);
template cudaError_t batch::launch_tiled_iterations<float>(const FusedView<float>&, const FusedView<float>&,
                                                           const Physics&, const PersistArgs&, int, int, int, bool,
                                                           cudaStream_t);

}  // namespace e3d
