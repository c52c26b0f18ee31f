// Tensor-map x coordinates count 8-byte words: a tile row is 16 words (128 bytes) whatever the
// storage type, so tile xt starts at word 16*xt.
// TMA-staged versions of the strided passes (y pencils; z pencils with the dyadic Green or the curl).
// Same arithmetic as k_y / k_zg in fm_passes.cuh; the data path goes through swizzled shared-memory
// tiles loaded and stored by the tensor memory accelerator (see fm_tma.cuh).
//
// Pipeline: a persistent CTA walks its tiles i = blockIdx.x, blockIdx.x + gridDim.x, ... (tiles of
// inactive right-hand sides skipped).  Thread 0 keeps NST loads in flight: after it has stored tile i
// from stage s (and the store has read the stage) it issues the load of tile i + NST into stage s.
// Every consumer warp waits on the stage's "full" barrier; each warp arrives on the stage's "done"
// barrier after writing its pencils back, and thread 0 waits on "done" before storing.
#pragma once
#include "fm_passes.cuh"
#include "fm_tma.cuh"

namespace fm {

// Shared-memory carve-up shared by the host launcher and the kernels.
template <int TILE_BYTES, int NST, int EXB, int TABB>
struct TmaSmem {
  static constexpr int tiles = 0;                                 // 1024-aligned
  static constexpr int ex = NST * TILE_BYTES;                     // exchange buffers
  static constexpr int tab = ex + ((EXB + 15) / 16) * 16;         // twiddles / ramps
  static constexpr int bars = tab + ((TABB + 15) / 16) * 16;      // 2*NST mbarriers
  static constexpr int total = bars + 2 * NST * 8 + 1024;         // + alignment slack
};

template <typename S, typename R, int L>
struct YTmaCfg {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P = Plan<L, R>;
  static constexpr int TX = 128 / (int)sizeof(TS);
  static constexpr int PW = 32 / P::TP;
  static constexpr int CW = (TX / PW) < 4 ? (TX / PW) : 4;
  static constexpr int ROUNDS = TX / (CW * PW);
  static constexpr int TILE = L * 128;
  static constexpr int NST = TILE <= 32768 ? 3 : 2;  // three stages leave room for three CTAs per SM
  static constexpr int STRIDE = PencilStride<L, T, P::TP, true>::v;
  using SM = TmaSmem<TILE, NST, CW * PW * STRIDE * (int)sizeof(T), L * (int)sizeof(T)>;
  static constexpr int THREADS = CW * 32;
};

// next tile of this CTA at or after `tile` whose right-hand side is active (ntiles if none)
__device__ __forceinline__ long long next_active(long long tile, long long ntiles, long long per_rhs,
                                                 const int* __restrict__ active) {
  while (tile < ntiles && active && !active[(int)(tile / per_rhs)]) tile += gridDim.x;
  return tile;
}

template <typename S, typename R, int L, int DIR>
__global__ void __launch_bounds__(YTmaCfg<S, R, L>::THREADS)
    k_y_tma(Dims d, const __grid_constant__ CUtensorMap tm_in, const __grid_constant__ CUtensorMap tm_out,
            const cplx<R>* __restrict__ twy, const cplx<R>* __restrict__ rampy, const int* __restrict__ active,
            int* __restrict__ err) {
  using C = YTmaCfg<S, R, L>;
  using T = typename C::T;
  using TS = typename C::TS;
  using P_ = typename C::P;
  constexpr int E = P_::E, TP = P_::TP, PW = C::PW, CW = C::CW, NST = C::NST, TX = C::TX;
  constexpr int BOX = L > 256 ? 256 : L;
  extern __shared__ unsigned char smraw_[];
  unsigned char* sm0 = (unsigned char*)(((uintptr_t)smraw_ + 1023) & ~(uintptr_t)1023);
  unsigned char* tiles = sm0 + C::SM::tiles;
  T* ex = reinterpret_cast<T*>(sm0 + C::SM::ex);
  T* tw = reinterpret_cast<T*>(sm0 + C::SM::tab);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm0 + C::SM::bars);
  uint64_t* done = full + NST;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xtiles = d.nx / TX;
  const long long per_rhs = (long long)xtiles * d.nz * 3;
  const long long ntiles = per_rhs * d.nb;
  load_table(tw, twy + (DIR < 0 ? 0 : L), L);
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(full + s, 1);
      mbar_init(done + s, CW);
    }
    fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](long long tile, int s) {
    const int xt = (int)(tile % xtiles);
    const int zcb = (int)(tile / xtiles);
    mbar_expect_tx(full + s, C::TILE);
    for (int k = 0; k < L / BOX; ++k)
      tma_load_3d(tiles + s * C::TILE + k * BOX * 128, &tm_in, full + s, xt * 16, k * BOX, zcb);
  };
  long long ld = next_active(blockIdx.x, ntiles, per_rhs, active);  // load cursor (thread 0)
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST && ld < ntiles; ++s) {
      issue(ld, s);
      ld = next_active(ld + gridDim.x, ntiles, per_rhs, active);
    }
  }
  const int p = lane / TP, t = lane % TP;  // t-fastest: consecutive rows across lanes
  T* sm = ex + (warp * PW + p) * C::STRIDE;
  int it = 0;
  bool ok = true;
  for (long long tile = next_active(blockIdx.x, ntiles, per_rhs, active); tile < ntiles;
       tile = next_active(tile + gridDim.x, ntiles, per_rhs, active)) {
    const int xt = (int)(tile % xtiles);
    const int zcb = (int)(tile / xtiles);
    const int s = it % NST;
    const uint32_t ph = (it / NST) & 1;
    if (!mbar_wait(full + s, ph, err, 13)) { ok = false; break; }
    unsigned char* tl = tiles + s * C::TILE;
#pragma unroll 1
    for (int rd = 0; rd < C::ROUNDS; ++rd) {
      const int xl = rd * CW * PW + warp * PW + p;
      T v[E];
      if constexpr (DIR < 0) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int y = lay_idx<L, E, P_::R0>(t, e);
          T a = cv<T>(*tile_at<TS>(tl, y, xl));
          if (rampy) a = cmul(a, rampy[y]);
          v[e] = a;
        }
        fft_fwd_plan<-1, P_>(v, sm, tw, t);
        __syncwarp();
#pragma unroll
        for (int e = 0; e < E; ++e) *tile_at<TS>(tl, lay_idx<L, E, P_::RL>(t, e), xl) = cv<TS>(v[e]);
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = cv<T>(*tile_at<TS>(tl, lay_idx<L, E, P_::RL>(t, e), xl));
        fft_rev_plan<+1, P_>(v, sm, tw, t);
        __syncwarp();
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int y = lay_idx<L, E, P_::R0>(t, e);
          T a = v[e];
          if (rampy) a = cmul(a, cconj(rampy[y]));
          *tile_at<TS>(tl, y, xl) = cv<TS>(a);
        }
      }
      __syncwarp();
    }
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive(done + s);
    if (threadIdx.x == 0) {
      if (!mbar_wait(done + s, ph, err, 14)) { ok = false; break; }
      for (int k = 0; k < L / BOX; ++k) tma_store_3d(&tm_out, tl + k * BOX * 128, xt * 16, k * BOX, zcb);
      bulk_commit();
      bulk_wait_read0();
      if (ld < ntiles) {
        issue(ld, s);
        ld = next_active(ld + gridDim.x, ntiles, per_rhs, active);
      }
    }
    ++it;
  }
  if (threadIdx.x == 0) {
    if (!ok) {
      // drain the loads this thread issued but nobody consumed (bounded waits)
      for (int k = 0; k < NST; ++k) mbar_wait(full + ((it + k) % NST), ((it + k) / NST) & 1, err, 15);
    }
    bulk_wait0();
  }
}

// ---------------------------------------------------------------------------
// z pass: tile = TX x-pencils (128-byte rows) x Lz x 3 components at fixed (y, b).
// ---------------------------------------------------------------------------
template <typename S, typename R, int L, int MODE>
struct ZTmaCfg {
  using T = cplx<R>;
  using TS = cplx<S>;
  static constexpr int LF = (MODE == ZMODE_AVG2) ? 2 * L : L;
  using P = Plan<LF, R>;
  static constexpr int TX = 128 / (int)sizeof(TS);
  static constexpr int PW = 32 / P::TP;
  static constexpr int CW = (TX / PW) < 8 ? (TX / PW) : 8;
  static constexpr int ROUNDS = TX / (CW * PW);
  static constexpr int TILE = 3 * L * 128;
  static constexpr int NST = TILE <= 32768 ? 3 : 2;
  static constexpr int STRIDE = PencilStride<LF, T, P::TP, true>::v;
  // exchange buffers per pencil: the three components of a length-256 transform run stage by stage together
  // (their exchanges overlap), each with its own buffer; shorter transforms run one component at a time
  static constexpr int NCX = LF >= 256 ? 3 : 1;
  using SM = TmaSmem<TILE, NST, CW * PW * NCX * STRIDE * (int)sizeof(T), (2 * LF + L) * (int)sizeof(T)>;
  static constexpr int THREADS = CW * 32;
};

template <typename S, typename R, int L, int MODE>
__global__ void __launch_bounds__(ZTmaCfg<S, R, L, MODE>::THREADS)
    k_zg_tma(Dims d, const __grid_constant__ CUtensorMap tm_in, const __grid_constant__ CUtensorMap tm_out,
             GreenParams gp, const cplx<R>* __restrict__ twz, const cplx<R>* __restrict__ rz,
             const int* __restrict__ active, int* __restrict__ err) {
  using C = ZTmaCfg<S, R, L, MODE>;
  using T = typename C::T;
  using TS = typename C::TS;
  using P_ = typename C::P;
  constexpr int LF = C::LF, E = P_::E, TP = P_::TP, PW = C::PW, CW = C::CW, NST = C::NST, TX = C::TX;
  extern __shared__ unsigned char smraw_[];
  unsigned char* sm0 = (unsigned char*)(((uintptr_t)smraw_ + 1023) & ~(uintptr_t)1023);
  unsigned char* tiles = sm0 + C::SM::tiles;
  T* ex = reinterpret_cast<T*>(sm0 + C::SM::ex);
  T* tw = reinterpret_cast<T*>(sm0 + C::SM::tab);
  T* twr = tw + LF;
  T* rtab = twr + LF;
  uint64_t* full = reinterpret_cast<uint64_t*>(sm0 + C::SM::bars);
  uint64_t* done = full + NST;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xtiles = d.nx / TX;
  const long long per_rhs = (long long)xtiles * d.ny;
  const long long ntiles = per_rhs * d.nb;
  load_table(tw, twz, 2 * LF);
  if (rz) load_table(rtab, rz, L);
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; ++s) {
      mbar_init(full + s, 1);
      mbar_init(done + s, CW);
    }
    fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](long long tile, int s) {
    const int xt = (int)(tile % xtiles);
    const long long yb = tile / xtiles;
    mbar_expect_tx(full + s, C::TILE);
    tma_load_4d(tiles + s * C::TILE, &tm_in, full + s, xt * 16, (int)(yb % d.ny), 0, 3 * (int)(yb / d.ny));
  };
  long long ld = next_active(blockIdx.x, ntiles, per_rhs, active);
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST && ld < ntiles; ++s) {
      issue(ld, s);
      ld = next_active(ld + gridDim.x, ntiles, per_rhs, active);
    }
  }
  const int p = lane / TP, t = lane % TP;
  constexpr int NCX = C::NCX, SMS = C::STRIDE;
  T* sm = ex + (warp * PW + p) * NCX * SMS;
  const R ksr = (R)gp.ksq_re;
  const T sc = mk((R)gp.scale_re, (R)gp.scale_im);
  int it = 0;
  bool ok = true;
  for (long long tile = next_active(blockIdx.x, ntiles, per_rhs, active); tile < ntiles;
       tile = next_active(tile + gridDim.x, ntiles, per_rhs, active)) {
    const int xt = (int)(tile % xtiles);
    const long long yb = tile / xtiles;
    const int y = (int)(yb % d.ny), b = (int)(yb / d.ny);
    const int s = it % NST;
    const uint32_t ph = (it / NST) & 1;
    if (!mbar_wait(full + s, ph, err, 23)) { ok = false; break; }
    unsigned char* tl = tiles + s * C::TILE;
    const R ksi = gp.ksq_im_b ? (R)gp.ksq_im_b[b] : (R)gp.ksq_im;
    const R kden = ksr * ksr + ksi * ksi;
    const T iks = mk(ksr / kden, -ksi / kden);
#pragma unroll 1
    for (int rd = 0; rd < C::ROUNDS; ++rd) {
      const int xl = rd * CW * PW + warp * PW + p;
      const int x = xt * TX + xl;
      T v[3][E];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int z = lay_idx<LF, E, P_::R0>(t, e);
          T a = czero<T>();
          if (MODE != ZMODE_AVG2 || z < L) {
            a = cv<T>(*tile_at<TS>(tl, c * L + z, xl));
            if (MODE != ZMODE_CURL && rz) a = cmul(a, rtab[z]);
          }
          v[c][e] = a;
        }
        if constexpr (NCX == 1) {
          fft_fwd_plan<-1, P_>(v[c], sm, tw, t);
          __syncwarp();
        }
      }
      if constexpr (NCX == 3) {
        fft_fwd_plan_n<-1, P_, 3, SMS>(v, sm, tw, t);
        __syncwarp();
      }
      R kx, ky;
      if (MODE == ZMODE_CURL) {
        kx = (R)gp.dk[0] * kidx_curl<R>(x, d.nx);
        ky = (R)gp.dk[1] * kidx_curl<R>(y, d.ny);
      } else {
        kx = (R)gp.dk[0] * (kidx_green<R>(x, d.nx) + (R)gp.shift[0]);
        ky = (R)gp.dk[1] * (kidx_green<R>(y, d.ny) + (R)gp.shift[1]);
      }
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int m = lay_idx<LF, E, P_::RL>(t, e);
        R kz;
        if constexpr (MODE == ZMODE_AVG2) {
          if ((m & 1) == 0) kz = (R)gp.dk[2] * (kidx_green<R>(m >> 1, L) + (R)gp.shift[2]);
          else kz = (R)gp.dk[2] * (kidx_green<R>(((m + 1) >> 1) % L, L) - (R)gp.shift[2]);
        } else if constexpr (MODE == ZMODE_ONE) {
          kz = (R)gp.dk[2] * (kidx_green<R>(m, L) + (R)gp.shift[2]);
        } else {
          kz = (R)gp.dk[2] * kidx_curl<R>(m, L);
        }
        T e1 = v[0][e], e2 = v[1][e], e3 = v[2][e];
        if constexpr (MODE == ZMODE_CURL) {
          const T isc = cmul_i<1>(sc);
          v[0][e] = cmul(csub(cscale(e3, ky), cscale(e2, kz)), isc);
          v[1][e] = cmul(csub(cscale(e1, kz), cscale(e3, kx)), isc);
          v[2][e] = cmul(csub(cscale(e2, kx), cscale(e1, ky)), isc);
        } else {
          T kE = cmul(cadd(cadd(cscale(e1, kx), cscale(e2, ky)), cscale(e3, kz)), iks);
          const R k2 = kx * kx + ky * ky + kz * kz;
          const R dr = k2 - ksr, di = -ksi;
          const R dd = dr * dr + di * di;
          const R rdd = R(1) / dd;  // one division for both parts of 1 / (k^2 - ks)
          const T f = cmul(sc, mk(dr * rdd, -di * rdd));
          v[0][e] = cmul(csub(e1, cscale(kE, kx)), f);
          v[1][e] = cmul(csub(e2, cscale(kE, ky)), f);
          v[2][e] = cmul(csub(e3, cscale(kE, kz)), f);
        }
      }
      if constexpr (NCX == 3) {
        fft_rev_plan_n<+1, P_, 3, SMS>(v, sm, twr, t);
        __syncwarp();
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if constexpr (NCX == 1) {
          fft_rev_plan<+1, P_>(v[c], sm, twr, t);
          __syncwarp();
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int z = lay_idx<LF, E, P_::R0>(t, e);
          if (MODE != ZMODE_AVG2 || z < L) {
            T a = v[c][e];
            if (MODE != ZMODE_CURL && rz) a = cmul(a, cconj(rtab[z]));
            *tile_at<TS>(tl, c * L + z, xl) = cv<TS>(a);
          }
        }
      }
      __syncwarp();
    }
    fence_proxy_async();
    __syncwarp();
    if (lane == 0) mbar_arrive(done + s);
    if (threadIdx.x == 0) {
      if (!mbar_wait(done + s, ph, err, 24)) { ok = false; break; }
      tma_store_4d(&tm_out, tl, xt * 16, y, 0, 3 * b);
      bulk_commit();
      bulk_wait_read0();
      if (ld < ntiles) {
        issue(ld, s);
        ld = next_active(ld + gridDim.x, ntiles, per_rhs, active);
      }
    }
    ++it;
  }
  if (threadIdx.x == 0) {
    if (!ok) {
      for (int k = 0; k < NST; ++k) mbar_wait(full + ((it + k) % NST), ((it + k) / NST) & 1, err, 25);
    }
    bulk_wait0();
  }
}

}  // namespace fm
