// Launchers and host tables of the general-length passes (fm_generic.cuh), for the three storage /
// arithmetic pairs of the plans.
#include <algorithm>
#include <cmath>

#include "fm_generic.h"
#include "fm_tables.h"

namespace fm {

GenAxisTables gen_axis_tables(int n) {
  GenAxisTables t;
  t.n = n;
  t.m = gen_fft_length(n);
  const int m = t.m;
  // (the stage twiddles of length m depend on the arithmetic type's radix split: the caller takes them from
  // twiddles<R>(m))
  if (m == n) return t;
  for (int dir = 0; dir < 2; ++dir) {
    const double sg = dir == 0 ? -1.0 : 1.0;
    t.chirp[dir].resize(n);
    for (int k = 0; k < n; ++k) {
      // c_k = exp(sg i pi k^2 / n), with k^2 reduced mod 2n so the angle stays small
      const long long q = ((long long)k * k) % (2LL * n);
      const double a = sg * M_PI * (double)q / (double)n;
      t.chirp[dir][k] = std::complex<double>(std::cos(a), std::sin(a));
    }
    // b (length m): conj(c_j) at j and at m - j (j < n), zero elsewhere; kern = DFT_m(b) / m
    std::vector<std::complex<double>> b(m, 0.0);
    for (int j = 0; j < n; ++j) {
      b[j] = std::conj(t.chirp[dir][j]);
      if (j > 0) b[m - j] = std::conj(t.chirp[dir][j]);
    }
    t.kern[dir].assign(m, 0.0);
    for (int k = 0; k < m; ++k) {
      std::complex<double> s = 0.0;
      for (int j = 0; j < m; ++j) {
        if (b[j] == 0.0) continue;
        const long long q = ((long long)j * k) % m;
        const double a = -2.0 * M_PI * (double)q / (double)m;
        s += b[j] * std::complex<double>(std::cos(a), std::sin(a));
      }
      t.kern[dir][k] = s / (double)m;
    }
  }
  return t;
}

template <typename K>
static void gen_allow_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static unsigned gen_blocks(long long work) {
  return (unsigned)std::max<long long>(1, std::min<long long>((work + 255) / 256, 148LL * 32));
}

template <typename S, typename R, int M, int DIR>
static cudaError_t gen_axis_M(const Dims& d, int axis, const void* in, void* out, const GenAxis& ax, const int* act,
                              cudaStream_t st) {
  using T = cplx<R>;
  using P_ = Plan<M, R>;
  constexpr int PW = 32 / P_::TP;
  constexpr int W = 8;
  const long long pencils = d.n / ax.n * 3 * d.nb;
  const long long warps = (pencils + PW - 1) / PW;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(2 * M + W * PW * PencilStride<M, T, P_::TP, true>::v) * sizeof(T);
  gen_allow_smem(k_gen_axis<S, R, M, DIR>, smem);
  k_gen_axis<S, R, M, DIR><<<blocks, W * 32, smem, st>>>(d, axis, (const cplx<S>*)in, (cplx<S>*)out, ax, act);
  return cudaGetLastError();
}

template <typename S, typename R>
cudaError_t launch_gen_axis(const Dims& d, int axis, int dir, const void* in, void* out, const GenAxis& ax,
                            const int* act, cudaStream_t st) {
#define FM_GEN_AXIS(MM)                                                               \
  case MM:                                                                            \
    return dir < 0 ? gen_axis_M<S, R, MM, -1>(d, axis, in, out, ax, act, st)          \
                   : gen_axis_M<S, R, MM, +1>(d, axis, in, out, ax, act, st);
  switch (ax.m) {
    FM_GEN_AXIS(8)
    FM_GEN_AXIS(16)
    FM_GEN_AXIS(32)
    FM_GEN_AXIS(64)
    FM_GEN_AXIS(128)
    FM_GEN_AXIS(256)
    FM_GEN_AXIS(512)
    default:
      return cudaErrorNotSupported;
  }
#undef FM_GEN_AXIS
}

template <typename S, typename R>
cudaError_t launch_gen_pre(const Dims& d, int pro, const void* in, const void* V, const double* rs, const GenRamps& rp,
                           void* out, const int* act, cudaStream_t st, VecTab vt) {
  const unsigned bl = gen_blocks(3 * d.n * d.nb);
  if (pro == PRO_COPY)
    k_gen_pre<S, R, PRO_COPY><<<bl, 256, 0, st>>>(d, (const cplx<S>*)in, (const cplx<S>*)V, rs, rp, (cplx<S>*)out, act, vt);
  else if (pro == PRO_V)
    k_gen_pre<S, R, PRO_V><<<bl, 256, 0, st>>>(d, (const cplx<S>*)in, (const cplx<S>*)V, rs, rp, (cplx<S>*)out, act, vt);
  else
    k_gen_pre<S, R, PRO_V_SCALE><<<bl, 256, 0, st>>>(d, (const cplx<S>*)in, (const cplx<S>*)V, rs, rp, (cplx<S>*)out, act,
                                                     vt);
  return cudaGetLastError();
}

template <typename S, typename R>
cudaError_t launch_gen_kspace(const Dims& d, int mode, void* f, const GreenParams& gp, const int* act, cudaStream_t st) {
  const unsigned bl = gen_blocks(d.n * d.nb);
  if (mode == ZMODE_CURL) k_gen_kspace<S, R, ZMODE_CURL><<<bl, 256, 0, st>>>(d, (cplx<S>*)f, gp, act);
  else k_gen_kspace<S, R, ZMODE_ONE><<<bl, 256, 0, st>>>(d, (cplx<S>*)f, gp, act);
  return cudaGetLastError();
}

template <typename S, typename R>
cudaError_t launch_gen_post(const Dims& d, int epi, const void* in, const void* V, const void* xv, const void* bv,
                            const double* rs, const EpiParams& ep, const GenRamps& rp, void* out, const int* act,
                            cudaStream_t st, VecTab vt) {
  using TS = cplx<S>;
  const unsigned bl = gen_blocks(3 * d.n * d.nb);
#define FM_GEN_POST(EE)                                                                                          \
  k_gen_post<S, R, EE><<<bl, 256, 0, st>>>(d, (const TS*)in, (const TS*)V, (const TS*)xv, (const TS*)bv, rs, ep, rp, \
                                           (TS*)out, act, vt)
  switch (epi) {
    case EPI_STORE: FM_GEN_POST(EPI_STORE); break;
    case EPI_OP: FM_GEN_POST(EPI_OP); break;
    case EPI_PREC_OP: FM_GEN_POST(EPI_PREC_OP); break;
    case EPI_PREC_RES: FM_GEN_POST(EPI_PREC_RES); break;
    default: return cudaErrorInvalidValue;
  }
#undef FM_GEN_POST
  return cudaGetLastError();
}

#define FM_GEN_INST(S, R)                                                                                          \
  template cudaError_t launch_gen_axis<S, R>(const Dims&, int, int, const void*, void*, const GenAxis&, const int*, \
                                             cudaStream_t);                                                       \
  template cudaError_t launch_gen_pre<S, R>(const Dims&, int, const void*, const void*, const double*,             \
                                            const GenRamps&, void*, const int*, cudaStream_t, VecTab);              \
  template cudaError_t launch_gen_kspace<S, R>(const Dims&, int, void*, const GreenParams&, const int*,            \
                                               cudaStream_t);                                                     \
  template cudaError_t launch_gen_post<S, R>(const Dims&, int, const void*, const void*, const void*, const void*, \
                                             const double*, const EpiParams&, const GenRamps&, void*, const int*,  \
                                             cudaStream_t, VecTab);
FM_GEN_INST(double, double)
FM_GEN_INST(float, double)
FM_GEN_INST(float, float)
#undef FM_GEN_INST

}  // namespace fm
