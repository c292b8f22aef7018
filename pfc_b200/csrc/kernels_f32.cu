// F32 instantiation of the relaxation kernels (kernels_impl.cuh).
#include "kernels_impl.cuh"

namespace pfcg {

template cudaError_t launch_xpass<float>(int, const XArgs<float>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_ypass<float>(int, const YArgs<float>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_kspace_energy<float>(const cplx<float>*, long long, const Model&, const Geom&, int, const double*,
                                               const double*, double*, double*, cudaStream_t);

template cudaError_t launch_ct_batch<float>(int, int, int, const void*, const int*, const int*, int, const LaunchCfg&,
                                           cudaStream_t);
template cudaError_t launch_generic_batch<float>(int, const void*, const int*, const int*, int, int, int, cudaStream_t);

template void prepare_batch_kernels<float>();

} // namespace pfcg
