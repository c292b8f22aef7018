// F32 instantiation of the relaxation kernels (kernels_impl.cuh).
#include "kernels_impl.cuh"

namespace pfcg {

template cudaError_t launch_xpass<float>(int, const XArgs<float>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_ypass<float>(int, const YArgs<float>&, const LaunchCfg&, cudaStream_t);
template cudaError_t launch_kspace_energy<float>(const cplx<float>*, long long, const Model&, const Geom&, int, const double*,
                                               const double*, double*, cudaStream_t);

} // namespace pfcg
