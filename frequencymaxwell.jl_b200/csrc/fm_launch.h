// Host-side launchers of the axis passes.  S is the storage type of the fields in
// HBM, R the arithmetic type in registers (S = R, or float storage with double
// arithmetic).  Each (S, R) pair is instantiated in its own translation unit.
#pragma once
#include <cuda_runtime.h>
#include "fm_passes.cuh"

namespace fm {

// Largest supported axis length and the largest z length with the averaged
// (length-2L) transform.
constexpr int AXIS_MAX = 512;
// axis lengths with an FFT plan: powers of two in [8, AXIS_MAX] and 96 (radices 8, 4, 3)
inline bool axis_supported(int n) { return (n >= 8 && n <= AXIS_MAX && (n & (n - 1)) == 0) || n == 96; }
constexpr int AXIS_MAX_AVG2 = 256;

template <typename S, typename R>
cudaError_t launch_xf(const Dims& d, int pro, const void* in, const void* V, const double* rhs_scale, const void* twx,
                      const void* rampx, void* out, const int* active, cudaStream_t st, VecTab vt = VecTab{});
template <typename S, typename R>
cudaError_t launch_y(const Dims& d, int dir, const void* in, const void* twy, const void* rampy, void* out,
                     const int* active, cudaStream_t st);
template <typename S, typename R>
cudaError_t launch_zg(const Dims& d, int mode, const void* in, const GreenParams& gp, const void* twz, const void* rz,
                      void* out, const int* active, cudaStream_t st);
template <typename S, typename R>
cudaError_t launch_xi(const Dims& d, int epi, const void* in, const void* V, const void* xv, const void* bv,
                      const double* rhs_scale, const EpiParams& ep, const void* twx, const void* rampx, void* out,
                      const int* active, cudaStream_t st, VecTab vt = VecTab{});
// XI with EPI_PREC_OP (no x ramp, contiguous batches) and the next application's XF (PRO_V) of its result:
// out = the operator result, out2 = the x-transformed V .* out
template <typename S, typename R>
cudaError_t launch_xi_xf(const Dims& d, const void* in, const void* V, const void* xv, const EpiParams& ep,
                         const void* twx, void* out, void* out2, const int* active, cudaStream_t st);

// TMA-staged y and z passes (fm_passes_tma.cuh).  They return cudaErrorNotSupported when the
// shape has no TMA variant (the caller then uses the register-only passes).  `err` receives a
// non-zero code if a pipeline wait timed out.
template <typename S, typename R>
cudaError_t launch_y_tma(const Dims& d, int dir, const void* in, const void* twy, const void* rampy, void* out,
                         const int* active, int* err, int sms, cudaStream_t st);
template <typename S, typename R>
cudaError_t launch_zg_tma(const Dims& d, int mode, const void* in, const GreenParams& gp, const void* twz,
                          const void* rz, void* out, const int* active, int* err, int sms, cudaStream_t st);

// pencils that share one warp for an axis of length L (y/z passes need nx to be a multiple)
template <typename R>
int pencils_per_warp(int L);

}  // namespace fm
