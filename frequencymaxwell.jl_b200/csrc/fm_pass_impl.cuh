// Launcher bodies for the axis passes; included once per precision.
#pragma once
#include "fm_launch.h"
#include "fm_passes_tma.cuh"

namespace fm {

template <typename K>
static void allow_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

constexpr int ROW_THREADS = 256;  // default threads per block of the row passes
constexpr int ZG_THREADS = ZG_WARPS * 32;
// threads per block of the x and y row passes: 128 or 256 (the tuning value in Dims), else the default
static inline int row_threads(const Dims& d) { return d.row_threads == 128 ? 128 : ROW_THREADS; }

template <typename S, typename R, int L, int PRO>
static cudaError_t xf_L(const Dims& d, const void* in, const void* V, const double* rs, const void* tw, const void* ramp,
                        void* out, const int* act, cudaStream_t st, const VecTab& vt) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP;
  const int W = row_threads(d) / 32;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long warps = rows / PW;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(L + W * PW * PencilStride<L, T, P_::TP, true>::v) * sizeof(T);
  allow_smem(k_xf<S, R, L, PRO>, smem);
  k_xf<S, R, L, PRO><<<blocks, W * 32, smem, st>>>(d, (const TS*)in, (const TS*)V, rs, (const T*)tw,
                                                         (const T*)ramp, (TS*)out, act, vt);
  return cudaGetLastError();
}

template <typename S, typename R, int L, int EPI>
static cudaError_t xi_L(const Dims& d, const void* in, const void* V, const void* xv, const void* bv, const double* rs,
                        const EpiParams& ep, const void* tw, const void* ramp, void* out, const int* act,
                        cudaStream_t st, const VecTab& vt) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP;
  const int W = row_threads(d) / 32;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long warps = rows / PW;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(L + W * PW * PencilStride<L, T, P_::TP, true>::v) * sizeof(T);
  allow_smem(k_xi<S, R, L, EPI>, smem);
  k_xi<S, R, L, EPI><<<blocks, W * 32, smem, st>>>(d, (const TS*)in, (const TS*)V, (const TS*)xv, (const TS*)bv,
                                                         rs, ep, (const T*)tw, (const T*)ramp, (TS*)out, act, vt);
  return cudaGetLastError();
}

template <typename S, typename R, int L>
static cudaError_t xi_xf_L(const Dims& d, const void* in, const void* V, const void* xv, const EpiParams& ep,
                           const void* tw, void* out, void* out2, const int* act, cudaStream_t st) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP;
  const int W = row_threads(d) / 32;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long warps = rows / PW;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  const size_t smem = (size_t)(2 * L + W * PW * PencilStride<L, T, P_::TP, true>::v) * sizeof(T);
  allow_smem(k_xi_xf<S, R, L>, smem);
  k_xi_xf<S, R, L><<<blocks, W * 32, smem, st>>>(d, (const TS*)in, (const TS*)V, (const TS*)xv, ep, (const T*)tw,
                                                 (TS*)out, (TS*)out2, act);
  return cudaGetLastError();
}

template <typename S, typename R, int L, int DIR>
static cudaError_t y_L(const Dims& d, const void* in, const void* tw, const void* ramp, void* out, const int* act,
                       cudaStream_t st) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int PW = 32 / P_::TP;
  const int W = row_threads(d) / 32;
  const long long warps = (long long)(d.nx / PW) * d.nz * 3 * d.nb;
  const unsigned blocks = (unsigned)((warps + W - 1) / W);
  // one pencil per warp and FP32 storage: four x-consecutive pencils per CTA, staged for coalesced rows
  if constexpr (PW == 1 && std::is_same<S, float>::value) {
    if (d.nx % YG_WARPS == 0) {
      const unsigned blocks_s = (unsigned)((warps + YG_WARPS - 1) / YG_WARPS);
      const size_t smem_s = (size_t)(L + YG_WARPS * PW * PencilStride<L, T, P_::TP, false>::v) * sizeof(T) +
                            (size_t)L * YG_WARPS * sizeof(TS);
      allow_smem(k_y<S, R, L, DIR, true>, smem_s);
      k_y<S, R, L, DIR, true><<<blocks_s, YG_WARPS * 32, smem_s, st>>>(d, (const TS*)in, (const T*)tw,
                                                                       (const T*)ramp, (TS*)out, act);
      return cudaGetLastError();
    }
  }
  const size_t smem = (size_t)(L + W * PW * PencilStride<L, T, P_::TP, false>::v) * sizeof(T);
  allow_smem(k_y<S, R, L, DIR>, smem);
  k_y<S, R, L, DIR><<<blocks, W * 32, smem, st>>>(d, (const TS*)in, (const T*)tw, (const T*)ramp, (TS*)out, act);
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
  // one pencil per warp and FP32 storage: stage the CTA's column block for coalesced loads and stores
  if constexpr (PW == 1 && std::is_same<S, float>::value) {
    if (d.nx % W == 0) {
      const size_t smem_s = smem + (size_t)3 * L * W * sizeof(TS);
      allow_smem(k_zg<S, R, L, MODE, true>, smem_s);
      k_zg<S, R, L, MODE, true><<<blocks, ZG_THREADS, smem_s, st>>>(d, (const TS*)in, gp, (const T*)tw, (const T*)rz,
                                                                    (TS*)out, act);
      return cudaGetLastError();
    }
  }
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
    case 96: return EXPR(96);                       \
    default: return cudaErrorInvalidValue;          \
  }

template <typename S, typename R>
cudaError_t launch_xf(const Dims& d, int pro, const void* in, const void* V, const double* rs, const void* tw,
                      const void* ramp, void* out, const int* act, cudaStream_t st, VecTab vt) {
#define XF_(LL, P) xf_L<S, R, LL, P>(d, in, V, rs, tw, ramp, out, act, st, vt)
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
                      const int* act, cudaStream_t st, VecTab vt) {
#define XI_(LL, E) xi_L<S, R, LL, E>(d, in, V, xv, bv, rs, ep, tw, ramp, out, act, st, vt)
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
cudaError_t launch_xi_xf(const Dims& d, const void* in, const void* V, const void* xv, const EpiParams& ep,
                         const void* tw, void* out, void* out2, const int* act, cudaStream_t st) {
#define XX(LL) xi_xf_L<S, R, LL>(d, in, V, xv, ep, tw, out, out2, act, st)
  FM_SWITCH_L(d.nx, XX, XX)
#undef XX
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

// ---- TMA tensor maps ----------------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// Field batch viewed as 8-byte elements (one complex64, or half a complex128).
// rank 3: (x, y, z*3*nb)  box (128 B, by, 1)      -- y pencils
// rank 4: (x, y, z, 3*nb) box (128 B, 1, bz, 3)   -- z pencils, all components
static bool make_map(CUtensorMap* m, void* base, const Dims& d, int esz, int rank, int box_y, int box_z) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const int w = esz / 8;  // 8-byte words per complex value
  cuuint64_t dims[4], strides[3];
  cuuint32_t box[4], es[4] = {1, 1, 1, 1};
  dims[0] = (cuuint64_t)d.nx * w;
  dims[1] = (cuuint64_t)d.ny;
  strides[0] = (cuuint64_t)d.nx * esz;
  strides[1] = (cuuint64_t)d.nx * d.ny * esz;
  box[0] = 16;
  if (rank == 3) {
    dims[2] = (cuuint64_t)d.nz * 3 * d.nb;
    box[1] = (cuuint32_t)box_y;
    box[2] = 1;
  } else {
    dims[2] = (cuuint64_t)d.nz;
    dims[3] = (cuuint64_t)3 * d.nb;
    strides[2] = (cuuint64_t)d.n * esz;
    box[1] = 1;
    box[2] = (cuuint32_t)box_z;
    box[3] = 3;
  }
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, (cuuint32_t)rank, base, dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <typename K>
static unsigned persistent_grid(K kern, int threads, size_t smem, long long ntiles, int sms, int cap = 0) {
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, threads, smem) != cudaSuccess || bps < 1) bps = 1;
  if (cap > 0 && bps > cap) bps = cap;  // tuning: fewer persistent CTAs per SM
  long long g = (long long)sms * bps;
  if (g > ntiles) g = ntiles;
  return (unsigned)(g < 1 ? 1 : g);
}

template <typename S, typename R, int L, int DIR>
static cudaError_t y_tma_L(const Dims& d, const void* in, const void* tw, const void* ramp, void* out, const int* act,
                           int* err, int sms, cudaStream_t st) {
  using C = YTmaCfg<S, R, L>;
  if (d.nx % C::TX) return cudaErrorNotSupported;
  CUtensorMap mi, mo;
  const int box = L > 256 ? 256 : L;
  if (!make_map(&mi, const_cast<void*>(in), d, (int)sizeof(cplx<S>), 3, box, 1) ||
      !make_map(&mo, out, d, (int)sizeof(cplx<S>), 3, box, 1))
    return cudaErrorNotSupported;
  const size_t smem = C::SM::total;
  allow_smem(k_y_tma<S, R, L, DIR>, smem);
  const long long ntiles = (long long)(d.nx / C::TX) * d.nz * 3 * d.nb;
  const unsigned grid = persistent_grid(k_y_tma<S, R, L, DIR>, C::THREADS, smem, ntiles, sms, d.tma_ctas);
  k_y_tma<S, R, L, DIR><<<grid, C::THREADS, smem, st>>>(d, mi, mo, (const cplx<R>*)tw + 0, (const cplx<R>*)ramp, act,
                                                         err);
  return cudaGetLastError();
}

template <typename S, typename R, int L, int MODE>
static cudaError_t zg_tma_L(const Dims& d, const void* in, const GreenParams& gp, const void* tw, const void* rz,
                            void* out, const int* act, int* err, int sms, cudaStream_t st) {
  using C = ZTmaCfg<S, R, L, MODE>;
  static_assert(C::SM::total <= 232448, "z pass shared memory above the 227 KB a CTA can have");
  if (d.nx % C::TX) return cudaErrorNotSupported;
  CUtensorMap mi, mo;
  if (!make_map(&mi, const_cast<void*>(in), d, (int)sizeof(cplx<S>), 4, 1, L) ||
      !make_map(&mo, out, d, (int)sizeof(cplx<S>), 4, 1, L))
    return cudaErrorNotSupported;
  const long long ntiles = (long long)(d.nx / C::TX) * d.ny * d.nb;
  const size_t smem = C::SM::total;
  allow_smem(k_zg_tma<S, R, L, MODE>, smem);
  const unsigned grid = persistent_grid(k_zg_tma<S, R, L, MODE>, C::THREADS, smem, ntiles, sms, d.tma_ctas);
  k_zg_tma<S, R, L, MODE><<<grid, C::THREADS, smem, st>>>(d, mi, mo, gp, (const cplx<R>*)tw, (const cplx<R>*)rz, act,
                                                           err);
  return cudaGetLastError();
}

template <typename S, typename R>
cudaError_t launch_y_tma(const Dims& d, int dir, const void* in, const void* tw, const void* ramp, void* out,
                         const int* act, int* err, int sms, cudaStream_t st) {
  // the table argument is the [forward | reversed] pair; the kernel picks its half
#define YT(LL) (dir < 0 ? y_tma_L<S, R, LL, -1>(d, in, tw, ramp, out, act, err, sms, st) \
                        : y_tma_L<S, R, LL, +1>(d, in, tw, ramp, out, act, err, sms, st))
  switch (d.ny) {
    case 96: return YT(96);
    case 32: return YT(32);
    case 64: return YT(64);
    case 128: return YT(128);
    case 256: return YT(256);
    default: return cudaErrorNotSupported;
  }
#undef YT
}

template <typename S, typename R>
cudaError_t launch_zg_tma(const Dims& d, int mode, const void* in, const GreenParams& gp, const void* tw,
                          const void* rz, void* out, const int* act, int* err, int sms, cudaStream_t st) {
#define ZT(LL, M) zg_tma_L<S, R, LL, M>(d, in, gp, tw, rz, out, act, err, sms, st)
  if (mode == ZMODE_AVG2) {
    switch (d.nz) {
      case 32: return ZT(32, ZMODE_AVG2);
      case 64: return ZT(64, ZMODE_AVG2);
      case 128: return ZT(128, ZMODE_AVG2);
      default: return cudaErrorNotSupported;
    }
  }
  if (mode == ZMODE_ONE) {
    switch (d.nz) {
      case 32: return ZT(32, ZMODE_ONE);
      case 64: return ZT(64, ZMODE_ONE);
      case 128: return ZT(128, ZMODE_ONE);
      default: return cudaErrorNotSupported;
    }
  }
  switch (d.nz) {
    case 32: return ZT(32, ZMODE_CURL);
    case 64: return ZT(64, ZMODE_CURL);
    case 128: return ZT(128, ZMODE_CURL);
    default: return cudaErrorNotSupported;
  }
#undef ZT
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
    case 96: return 32 / Plan<96, R>::TP;
    default: return 0;
  }
}

}  // namespace fm
