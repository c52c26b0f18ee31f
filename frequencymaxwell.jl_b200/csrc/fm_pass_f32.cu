// Axis-pass launchers instantiated for storage float, arithmetic float.
#include "fm_pass_impl.cuh"

namespace fm {
template cudaError_t launch_xf<float, float>(const Dims&, int, const void*, const void*, const double*, const void*,
                                      const void*, void*, const int*, cudaStream_t, VecTab);
template cudaError_t launch_y<float, float>(const Dims&, int, const void*, const void*, const void*, void*, const int*,
                                     cudaStream_t);
template cudaError_t launch_zg<float, float>(const Dims&, int, const void*, const GreenParams&, const void*, const void*,
                                      void*, const int*, cudaStream_t);
template cudaError_t launch_xi<float, float>(const Dims&, int, const void*, const void*, const void*, const void*,
                                      const double*, const EpiParams&, const void*, const void*, void*, const int*,
                                      cudaStream_t, VecTab);
template int pencils_per_warp<float>(int);
template cudaError_t launch_xi_xf<float, float>(const Dims&, const void*, const void*, const void*, const EpiParams&,
                                         const void*, void*, void*, const int*, cudaStream_t);
template cudaError_t launch_y_tma<float, float>(const Dims&, int, const void*, const void*, const void*, void*,
                                          const int*, int*, int, cudaStream_t);
template cudaError_t launch_zg_tma<float, float>(const Dims&, int, const void*, const GreenParams&, const void*,
                                          const void*, void*, const int*, int*, int, cudaStream_t);
}  // namespace fm
