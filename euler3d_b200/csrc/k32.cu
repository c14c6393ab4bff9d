// FP32 instantiations of the single-case fused path (multiply-add contraction
// allowed); the FP32 batch kernels are in k32b.cu.
#include "launch_common.cuh"

namespace e3d {

template void launch_halo<float>(int, const int*, const int*, int, float*, float*, cudaStream_t);
template void launch_halo_pack<float>(int, const int*, int, const float*, float*, cudaStream_t);
template void launch_halo_unpack<float>(int, const int*, int, const float*, float*, float*, cudaStream_t);
template void launch_reduce<float>(const ReduceArgs&, const float*, const float*, const float*, cudaStream_t);
template void launch_recon<float>(const FusedView<float>&, const Physics&, int, int, bool, int, cudaStream_t);
template void launch_start<float>(const FusedView<float>&, const Physics&, int, cudaStream_t);
template void launch_flux_update<float>(const FusedView<float>&, const Physics&, int, bool, double, double, int, int,
                                        cudaStream_t);


}  // namespace e3d
