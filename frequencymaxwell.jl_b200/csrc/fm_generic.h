// Host-side launchers and tables of the general-length passes (fm_generic.cuh).
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <vector>

#include "fm_generic.cuh"

namespace fm {

// Axis lengths the general passes take: powers of two in [8, 512] run the FFT directly; any length n in
// [1, 256] runs Bluestein's algorithm with a power-of-two FFT of length >= max(8, 2n - 1).
constexpr int GEN_AXIS_MAX = 256;
inline bool gen_axis_supported(int n) { return (n >= 1 && n <= GEN_AXIS_MAX) || (n >= 8 && n <= 512 && (n & (n - 1)) == 0); }
inline int gen_fft_length(int n) {
  if (n >= 8 && n <= 512 && (n & (n - 1)) == 0) return n;
  int m = 8;
  while (m < 2 * n - 1) m <<= 1;
  return m;
}

// FP64 host tables of one axis: twiddles of the FFT length, and for Bluestein lengths the chirps and the
// transformed convolution kernels of both directions (see GenAxis).
struct GenAxisTables {
  int n = 0, m = 0;
  std::vector<std::complex<double>> tw, chirp[2], kern[2];
};
GenAxisTables gen_axis_tables(int n);

template <typename S, typename R>
cudaError_t launch_gen_axis(const Dims& d, int axis, int dir, const void* in, void* out, const GenAxis& ax,
                            const int* act, cudaStream_t st);
template <typename S, typename R>
cudaError_t launch_gen_pre(const Dims& d, int pro, const void* in, const void* V, const double* rs, const GenRamps& rp,
                           void* out, const int* act, cudaStream_t st, VecTab vt = VecTab{});
template <typename S, typename R>
cudaError_t launch_gen_kspace(const Dims& d, int mode, void* f, const GreenParams& gp, const int* act, cudaStream_t st);
template <typename S, typename R>
cudaError_t launch_gen_post(const Dims& d, int epi, const void* in, const void* V, const void* xv, const void* bv,
                            const double* rs, const EpiParams& ep, const GenRamps& rp, void* out, const int* act,
                            cudaStream_t st, VecTab vt = VecTab{});

}  // namespace fm
