// F64 instantiation of the relaxation kernels (kernels_impl.cuh).
#include "kernels_impl.cuh"

namespace pfcg {

template cudaError_t launch_xpass<double>(int, const XArgs<double>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_ypass<double>(int, const YArgs<double>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_kspace_energy<double>(const cplx<double>*, long long, const Model&, const Geom&, int, const double*,
                                               const double*, double*, double*, cudaStream_t);

template cudaError_t launch_ct_batch<double>(int, int, int, const void*, const int*, const int*, int, const LaunchCfg&,
                                           cudaStream_t);
template cudaError_t launch_generic_batch<double>(int, const void*, const int*, const int*, int, int, int, cudaStream_t);

template void prepare_batch_kernels<double>();

} // namespace pfcg
