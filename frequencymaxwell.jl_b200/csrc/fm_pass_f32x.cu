// Axis-pass launchers instantiated for storage float, arithmetic double.
#include "fm_pass_impl.cuh"

namespace fm {
template cudaError_t launch_xf<float, double>(const Dims&, int, const void*, const void*, const double*, const void*,
                                      const void*, void*, const int*, cudaStream_t, VecTab);
template cudaError_t launch_y<float, double>(const Dims&, int, const void*, const void*, const void*, void*, const int*,
                                     cudaStream_t);
template cudaError_t launch_zg<float, double>(const Dims&, int, const void*, const GreenParams&, const void*, const void*,
                                      void*, const int*, cudaStream_t);
template cudaError_t launch_xi<float, double>(const Dims&, int, const void*, const void*, const void*, const void*,
                                      const double*, const EpiParams&, const void*, const void*, void*, const int*,
                                      cudaStream_t, VecTab);
template cudaError_t launch_xi_xf<float, double>(const Dims&, const void*, const void*, const void*, const EpiParams&,
                                         const void*, void*, void*, const int*, cudaStream_t);
template cudaError_t launch_y_tma<float, double>(const Dims&, int, const void*, const void*, const void*, void*,
                                          const int*, int*, int, cudaStream_t);
template cudaError_t launch_zg_tma<float, double>(const Dims&, int, const void*, const GreenParams&, const void*,
                                          const void*, void*, const int*, int*, int, cudaStream_t);
}  // namespace fm
