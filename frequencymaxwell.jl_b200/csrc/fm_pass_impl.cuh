// Launcher bodies for the axis passes; included once per precision.
#pragma once
#include "fm_launch.h"

namespace fm {

template <typename K>
static void allow_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

constexpr int ROW_THREADS = 256;
constexpr int ZG_THREADS = 128;

template <typename S, typename R, int L, int PRO>
static cudaError_t xf_L(const Dims& d, const void* in, const void* V, const double* rs, const void* tw, const void* ramp,
                        void* out, const int* act, cudaStream_t st) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP, W = ROW_THREADS / 32;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long warps = rows / PW;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(L + W * PW * PencilStride<L, T, P_::TP, true>::v) * sizeof(T);
  allow_smem(k_xf<S, R, L, PRO>, smem);
  k_xf<S, R, L, PRO><<<blocks, ROW_THREADS, smem, st>>>(d, (const TS*)in, (const TS*)V, rs, (const T*)tw,
                                                         (const T*)ramp, (TS*)out, act);
  return cudaGetLastError();
}

template <typename S, typename R, int L, int EPI>
static cudaError_t xi_L(const Dims& d, const void* in, const void* V, const void* xv, const void* bv, const double* rs,
                        const EpiParams& ep, const void* tw, const void* ramp, void* out, const int* act,
                        cudaStream_t st) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP, W = ROW_THREADS / 32;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long warps = rows / PW;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(L + W * PW * PencilStride<L, T, P_::TP, true>::v) * sizeof(T);
  allow_smem(k_xi<S, R, L, EPI>, smem);
  k_xi<S, R, L, EPI><<<blocks, ROW_THREADS, smem, st>>>(d, (const TS*)in, (const TS*)V, (const TS*)xv, (const TS*)bv,
                                                         rs, ep, (const T*)tw, (const T*)ramp, (TS*)out, act);
  return cudaGetLastError();
}

template <typename S, typename R, int L, int DIR>
static cudaError_t y_L(const Dims& d, const void* in, const void* tw, const void* ramp, void* out, const int* act,
                       cudaStream_t st) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP, W = ROW_THREADS / 32;
  const long long warps = (long long)(d.nx / PW) * d.nz * 3 * d.nb;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(L + W * PW * PencilStride<L, T, P_::TP, false>::v) * sizeof(T);
  allow_smem(k_y<S, R, L, DIR>, smem);
  k_y<S, R, L, DIR><<<blocks, ROW_THREADS, smem, st>>>(d, (const TS*)in, (const T*)tw, (const T*)ramp, (TS*)out, act);
  return cudaGetLastError();
}

template <typename S, typename R, int L, int MODE>
static cudaError_t zg_L(const Dims& d, const void* in, const GreenParams& gp, const void* tw, const void* rz, void* out,
                        const int* act, cudaStream_t st) {
  using T = cplx<R>;
  using TS = cplx<S>;
  constexpr int LF = (MODE == ZMODE_AVG2) ? 2 * L : L;
  using P_ = Plan<LF, R>;
  constexpr int PW = 32 / P_::TP, W = ZG_THREADS / 32;
  const long long warps = (long long)(d.nx / PW) * d.ny * d.nb;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(2 * LF + L + W * PW * PencilStride<LF, T, P_::TP, false>::v) * sizeof(T);
  allow_smem(k_zg<S, R, L, MODE>, smem);
  k_zg<S, R, L, MODE><<<blocks, ZG_THREADS, smem, st>>>(d, (const TS*)in, gp, (const T*)tw, (const T*)rz, (TS*)out,
                                                         act);
  return cudaGetLastError();
}

#define FM_SWITCH_L(L, EXPR8, EXPR)                 \
  switch (L) {                                      \
    case 8: return EXPR8(8);                        \
    case 16: return EXPR(16);                       \
    case 32: return EXPR(32);                       \
    case 64: return EXPR(64);                       \
    case 128: return EXPR(128);                     \
    case 256: return EXPR(256);                     \
    case 512: return EXPR(512);                     \
    default: return cudaErrorInvalidValue;          \
  }

template <typename S, typename R>
cudaError_t launch_xf(const Dims& d, int pro, const void* in, const void* V, const double* rs, const void* tw,
                      const void* ramp, void* out, const int* act, cudaStream_t st) {
#define XF_(LL, P) xf_L<S, R, LL, P>(d, in, V, rs, tw, ramp, out, act, st)
#define XF0(LL) XF_(LL, PRO_COPY)
#define XF1(LL) XF_(LL, PRO_V)
#define XF2(LL) XF_(LL, PRO_V_SCALE)
  if (pro == PRO_COPY) { FM_SWITCH_L(d.nx, XF0, XF0) }
  if (pro == PRO_V) { FM_SWITCH_L(d.nx, XF1, XF1) }
  FM_SWITCH_L(d.nx, XF2, XF2)
#undef XF_
#undef XF0
#undef XF1
#undef XF2
}

template <typename S, typename R>
cudaError_t launch_xi(const Dims& d, int epi, const void* in, const void* V, const void* xv, const void* bv,
                      const double* rs, const EpiParams& ep, const void* tw, const void* ramp, void* out,
                      const int* act, cudaStream_t st) {
#define XI_(LL, E) xi_L<S, R, LL, E>(d, in, V, xv, bv, rs, ep, tw, ramp, out, act, st)
#define XI0(LL) XI_(LL, EPI_STORE)
#define XI1(LL) XI_(LL, EPI_OP)
#define XI2(LL) XI_(LL, EPI_PREC_OP)
#define XI3(LL) XI_(LL, EPI_PREC_RES)
  if (epi == EPI_STORE) { FM_SWITCH_L(d.nx, XI0, XI0) }
  if (epi == EPI_OP) { FM_SWITCH_L(d.nx, XI1, XI1) }
  if (epi == EPI_PREC_OP) { FM_SWITCH_L(d.nx, XI2, XI2) }
  FM_SWITCH_L(d.nx, XI3, XI3)
#undef XI_
#undef XI0
#undef XI1
#undef XI2
#undef XI3
}

template <typename S, typename R>
cudaError_t launch_y(const Dims& d, int dir, const void* in, const void* tw, const void* ramp, void* out,
                     const int* act, cudaStream_t st) {
#define YF(LL) y_L<S, R, LL, -1>(d, in, tw, ramp, out, act, st)
#define YI(LL) y_L<S, R, LL, +1>(d, in, tw, ramp, out, act, st)
  if (dir < 0) { FM_SWITCH_L(d.ny, YF, YF) }
  FM_SWITCH_L(d.ny, YI, YI)
#undef YF
#undef YI
}

template <typename S, typename R>
cudaError_t launch_zg(const Dims& d, int mode, const void* in, const GreenParams& gp, const void* tw, const void* rz,
                      void* out, const int* act, cudaStream_t st) {
#define ZA(LL) zg_L<S, R, LL, ZMODE_AVG2>(d, in, gp, tw, rz, out, act, st)
#define ZO(LL) zg_L<S, R, LL, ZMODE_ONE>(d, in, gp, tw, rz, out, act, st)
#define ZC(LL) zg_L<S, R, LL, ZMODE_CURL>(d, in, gp, tw, rz, out, act, st)
  if (mode == ZMODE_AVG2) {
    switch (d.nz) {
      case 8: return ZA(8);
      case 16: return ZA(16);
      case 32: return ZA(32);
      case 64: return ZA(64);
      case 128: return ZA(128);
      case 256: return ZA(256);
      default: return cudaErrorInvalidValue;
    }
  }
  if (mode == ZMODE_ONE) { FM_SWITCH_L(d.nz, ZO, ZO) }
  FM_SWITCH_L(d.nz, ZC, ZC)
#undef ZA
#undef ZO
#undef ZC
}

template <typename R>
int pencils_per_warp(int L) {
  switch (L) {
    case 8: return 32 / Plan<8, R>::TP;
    case 16: return 32 / Plan<16, R>::TP;
    case 32: return 32 / Plan<32, R>::TP;
    case 64: return 32 / Plan<64, R>::TP;
    case 128: return 32 / Plan<128, R>::TP;
    case 256: return 32 / Plan<256, R>::TP;
    case 512: return 32 / Plan<512, R>::TP;
    default: return 0;
  }
}

}  // namespace fm
