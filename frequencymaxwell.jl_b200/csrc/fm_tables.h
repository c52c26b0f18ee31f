// Host-side construction of the FFT stage-twiddle tables and sub-pixel ramps (FP64, then cast to the
// arithmetic type of the kernels).
#pragma once
#include <cmath>
#include <complex>
#include <vector>

#include "fm_fft.cuh"

namespace fm {

using cd_t = std::complex<double>;

// Stage-twiddle table of one radix order (see fft_stage): entry (ns-1) + (q-1)*ns + k
// = exp(-2 pi i k q / (ns*R)) for each stage after the first.
inline void stage_table(std::vector<cd_t>& t, size_t off, const std::vector<int>& radices) {
  int ns = 1;
  for (size_t s = 0; s < radices.size(); ++s) {
    const int R = radices[s];
    if (s > 0)
      for (int q = 1; q < R; ++q)
        for (int k = 0; k < ns; ++k) {
          const double a = -2.0 * M_PI * (double)k * (double)q / ((double)ns * R);
          t[off + (ns - 1) + (size_t)(q - 1) * ns + k] = cd_t(std::cos(a), std::sin(a));
        }
    ns *= R;
  }
}

template <int L, typename R>
inline std::vector<int> radices_of() {
  using P_ = Plan<L, R>;
  std::vector<int> r{P_::R0};
  if (P_::R1) r.push_back(P_::R1);
  if (P_::R2) r.push_back(P_::R2);
  return r;
}

// [forward-order table | reversed-order table] for an FFT of length L in arithmetic type R
template <typename R>
inline std::vector<cd_t> twiddles(int L) {
  std::vector<int> r;
  switch (L) {
    case 8: r = radices_of<8, R>(); break;
    case 16: r = radices_of<16, R>(); break;
    case 32: r = radices_of<32, R>(); break;
    case 64: r = radices_of<64, R>(); break;
    case 128: r = radices_of<128, R>(); break;
    case 256: r = radices_of<256, R>(); break;
    case 512: r = radices_of<512, R>(); break;
    case 96: r = radices_of<96, R>(); break;
    default: break;
  }
  std::vector<cd_t> t(2 * (size_t)L, cd_t(1.0, 0.0));
  stage_table(t, 0, r);
  std::vector<int> rr(r.rbegin(), r.rend());
  stage_table(t, L, rr);
  return t;
}

// exp(sgn * 2 pi i * idx * s / L)
inline std::vector<cd_t> ramp(int L, double s, double sgn) {
  std::vector<cd_t> t(L);
  for (int k = 0; k < L; ++k) {
    double a = sgn * 2.0 * M_PI * (double)k * s / (double)L;
    t[k] = cd_t(std::cos(a), std::sin(a));
  }
  return t;
}

}  // namespace fm
