// Axis-pass launchers instantiated for double.
#include "fm_pass_impl.cuh"

namespace fm {
template cudaError_t launch_xf<double>(const Dims&, int, const void*, const void*, const double*, const void*, const void*,
                                      void*, const int*, cudaStream_t);
template cudaError_t launch_y<double>(const Dims&, int, const void*, const void*, const void*, void*, const int*,
                                     cudaStream_t);
template cudaError_t launch_zg<double>(const Dims&, int, const void*, const GreenParams&, const void*, const void*, void*,
                                      const int*, cudaStream_t);
template cudaError_t launch_xi<double>(const Dims&, int, const void*, const void*, const void*, const void*, const double*,
                                      const EpiParams&, const void*, const void*, void*, const int*, cudaStream_t);
template int pencils_per_warp<double>(int);
}  // namespace fm
