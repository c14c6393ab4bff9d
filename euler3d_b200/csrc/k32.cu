// FP32 instantiations of the fused path (multiply-add contraction allowed).
#include "launch_common.cuh"
#include "batch_launch.cuh"

namespace e3d {

template void launch_halo<float>(int, const int*, const int*, int, float*, float*, cudaStream_t);
template void launch_halo_pack<float>(int, const int*, int, const float*, float*, cudaStream_t);
template void launch_halo_unpack<float>(int, const int*, int, const float*, float*, float*, cudaStream_t);
template void launch_reduce<float>(const ReduceArgs&, const float*, const float*, const float*, cudaStream_t);
template void launch_recon<float>(const FusedView<float>&, const Physics&, int, int, bool, int, cudaStream_t);
template void launch_start<float>(const FusedView<float>&, const Physics&, int, cudaStream_t);
template void launch_flux_update<float>(const FusedView<float>&, const Physics&, int, bool, double, double, int, int,
                                        cudaStream_t);

template int batch::persistent_blocks_per_sm<float>(int, int, int, bool);
template cudaError_t batch::launch_persistent<float>(const FusedView<float>&, const FusedView<float>&, const Physics&,
                                              const PersistArgs&, int, int, int, bool, int, cudaStream_t);

template cudaError_t batch::launch_tiled_iterations<float>(const FusedView<float>&, const FusedView<float>&, const Physics&,
                                                    const PersistArgs&, int, int, int, bool, cudaStream_t);

}  // namespace e3d
