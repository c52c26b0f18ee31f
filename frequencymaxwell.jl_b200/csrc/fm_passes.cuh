// Axis passes of the dyadic-Green convolution and of the spectral curl.
//
// Field layout (column-major like the reference): element (x, y, z, c, b) of a
// batch of 3-component fields sits at x + nx*(y + ny*(z + nz*(c + 3*b))).
// One Green application G_avg(V.*x) runs as five passes, each reading and
// writing the batch once:
//   XF  x-rows   : psi = V.*x (prologue) -> forward FFT along x
//   YF  y-pencils: forward FFT along y
//   ZG  z-pencils: forward FFT along z -> 3x3 dyadic Green -> inverse FFT along z
//                  (both sub-pixel-shifted branches of the reference's average are
//                   produced by ONE length-2L transform of the zero-padded pencil)
//   YI  y-pencils: inverse FFT along y
//   XI  x-rows   : inverse FFT along x -> epilogue (operator / preconditioner / residual)
// Every pass keeps a pencil in registers (see fm_fft.cuh); warps are independent.
#pragma once
#include "fm_fft.cuh"

namespace fm {

// storage <-> compute conversion (identity when the types match)
template <typename To, typename From>
__device__ __forceinline__ To cv(From a) {
  if constexpr (std::is_same<To, From>::value) return a;
  else return mk((typename RealOf<To>::R)a.x, (typename RealOf<To>::R)a.y);
}

struct Dims {
  int nx, ny, nz, nb;
  long long n;           // nx*ny*nz
  long long vstride = 0; // potential of RHS b at V + b*vstride (0: one potential shared by all RHS)
  int row_threads = 256; // launch shape (tuning): threads per block of the x and y row passes (128 or 256)
  int tma_ctas = 0;      // launch shape (tuning): persistent CTAs per SM of the TMA passes (0: occupancy limit)
};

// Optional per-RHS vector pointers (RHS b's field starts at tab[b]); null -> contiguous batch.
struct VecTab {
  const void* const* in = nullptr;   // XF input / XI operator input x
  void* const* out = nullptr;        // XI output
};

// Warp-local exchange buffers: each warp owns PW pencils of STRIDE elements.
template <typename T, int STRIDE>
__device__ __forceinline__ T* warp_smem(T* base, int warp_in_cta, int pencils_per_warp, int p) {
  return base + ((size_t)warp_in_cta * pencils_per_warp + p) * STRIDE;
}

// Twiddle tables per FFT length are stored as [forward-order stage table (L) |
// reversed-order stage table (L)] (see fft_stage).

template <typename T>
__device__ __forceinline__ void load_table(T* dst, const T* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// XF: prologue + forward FFT along x.  One warp = P rows (y,z,b); a thread
// handles all 3 components of its row so V is loaded once.
// PRO: 0 copy, 1 multiply by V, 2 multiply by V and by a per-RHS real scale.
// ---------------------------------------------------------------------------
enum { PRO_COPY = 0, PRO_V = 1, PRO_V_SCALE = 2 };

template <typename S, typename R, int L, int PRO>
__global__ void __launch_bounds__(256, (L <= 128 && L != 96) ? 2 : 1) k_xf(Dims d, const cplx<S>* __restrict__ in, const cplx<S>* __restrict__ V,
                                            const double* __restrict__ rhs_scale, const cplx<R>* __restrict__ twx,
                                            const cplx<R>* __restrict__ rampx, cplx<S>* __restrict__ out,
                                            const int* __restrict__ active, VecTab vt) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int E = P_::E, TP = P_::TP, PW = 32 / TP;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tw = reinterpret_cast<T*>(smraw);
  T* ex = tw + L;
  load_table(tw, twx, L);
  __syncthreads();
  const int lane = threadIdx.x & 31, wic = threadIdx.x >> 5;
  const int p = lane / TP, t = lane % TP;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long row = ((long long)blockIdx.x * (blockDim.x >> 5) + wic) * PW + p;
  if (row >= rows) return;  // whole pencils exit together (rows is a multiple of PW)
  const int b = (int)(row / ((long long)d.ny * d.nz));
  if (active && !active[b]) return;
  const long long yz = row - (long long)b * d.ny * d.nz;
  T* sm = warp_smem<T, PencilStride<L, T, TP, true>::v>(ex, wic, PW, p);
  T vrow[E];
  if constexpr (PRO != PRO_COPY) {
#pragma unroll
    for (int e = 0; e < E; ++e) vrow[e] = cv<T>(V[b * d.vstride + yz * L + lay_idx<L, E, P_::R0>(t, e)]);
  }
  R s = R(1);
  if constexpr (PRO == PRO_V_SCALE) s = (R)rhs_scale[b];
  const cplx<S>* inb = vt.in ? (const cplx<S>*)vt.in[b] : in + (long long)b * 3 * d.n;
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    const long long base = ((long long)(c + 3 * b) * d.ny * d.nz + yz) * L;
    const long long rbase = ((long long)c * d.ny * d.nz + yz) * L;
    T v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = lay_idx<L, E, P_::R0>(t, e);
      T a = cv<T>(inb[rbase + x]);
      if constexpr (PRO != PRO_COPY) a = cmul(a, vrow[e]);
      if constexpr (PRO == PRO_V_SCALE) a = cscale(a, s);
      if (rampx) a = cmul(a, rampx[x]);
      v[e] = a;
    }
    fft_fwd_plan<-1, P_>(v, sm, tw, t);
#pragma unroll
    for (int e = 0; e < E; ++e) out[base + lay_idx<L, E, P_::RL>(t, e)] = cv<TS>(v[e]);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Y pass (forward DIR=-1 or inverse DIR=+1), plain.  One warp = P consecutive
// x columns at fixed (z, c, b); lane = t*P + p so consecutive lanes read
// consecutive x.
// ---------------------------------------------------------------------------
// STG (one pencil per warp only): the CTA's warps (YG_WARPS) take x-consecutive pencils of one (z, c, b) plane
// and the CTA stages the L x W block in shared memory with coalesced rows of W consecutive x values; the pencil
// slot is XOR-swizzled with bits 2.. of the row.  The launcher uses it when nx is a multiple of the warps per CTA.
constexpr int YG_WARPS = 4;
template <typename S, typename R, int L, int DIR, bool STG = false>
__global__ void __launch_bounds__(256) k_y(Dims d, const cplx<S>* __restrict__ in, const cplx<R>* __restrict__ twy,
                                           const cplx<R>* __restrict__ rampy, cplx<S>* __restrict__ out,
                                           const int* __restrict__ active) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int E = P_::E, TP = P_::TP, PW = 32 / TP;
  static_assert(!STG || PW == 1, "the staged y pass takes one pencil per warp");
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tw = reinterpret_cast<T*>(smraw);
  T* ex = tw + L;
  load_table(tw, twy + (DIR < 0 ? 0 : L), L);
  __syncthreads();
  const int lane = threadIdx.x & 31, wic = threadIdx.x >> 5;
  const int p = lane % PW, t = lane / PW;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + wic;
  const int xg = d.nx / PW;
  const long long total = (long long)xg * d.nz * 3 * d.nb;
  if (gw >= total) return;
  const int x = (int)(gw % xg) * PW + p;
  const long long zcb = gw / xg;  // z + nz*(c + 3b)
  const int b = (int)(zcb / (3LL * d.nz));
  if (active && !active[b]) return;
  const long long base = zcb * (long long)d.ny * d.nx + x;
  T* sm = warp_smem<T, PencilStride<L, T, TP, false>::v>(ex, wic, PW, p);
  constexpr int W = STG ? YG_WARPS : 1;
  static_assert(!STG || W == 4, "the swizzle assumes 4 pencils per row");
  auto tix = [](int r, int g) { return r * W + (g ^ ((r >> 2) & (W - 1))); };
  TS* tile = reinterpret_cast<TS*>(ex + (size_t)(blockDim.x >> 5) * PW * PencilStride<L, T, TP, false>::v);
  const long long cbase = base - wic;  // the CTA's first pencil
  if constexpr (STG) {
    for (int i = threadIdx.x; i < L * W; i += blockDim.x) {
      const int g = i % W, r = i / W;
      tile[tix(r, g)] = in[cbase + (long long)r * d.nx + g];
    }
    __syncthreads();
  }
  auto ld = [&](int y) -> T {
    if constexpr (STG) return cv<T>(tile[tix(y, wic)]);
    else return cv<T>(in[base + (long long)y * d.nx]);
  };
  auto st = [&](int y, T a) {
    if constexpr (STG) tile[tix(y, wic)] = cv<TS>(a);
    else out[base + (long long)y * d.nx] = cv<TS>(a);
  };
  T v[E];
  if constexpr (DIR < 0) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int y = lay_idx<L, E, P_::R0>(t, e);
      T a = ld(y);
      if (rampy) a = cmul(a, rampy[y]);
      v[e] = a;
    }
    fft_fwd_plan<-1, P_>(v, sm, tw, t);
#pragma unroll
    for (int e = 0; e < E; ++e) st(lay_idx<L, E, P_::RL>(t, e), v[e]);
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = ld(lay_idx<L, E, P_::RL>(t, e));
    fft_rev_plan<+1, P_>(v, sm, tw, t);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int y = lay_idx<L, E, P_::R0>(t, e);
      T a = v[e];
      if (rampy) a = cmul(a, cconj(rampy[y]));
      st(y, a);
    }
  }
  if constexpr (STG) {
    __syncthreads();
    for (int i = threadIdx.x; i < L * W; i += blockDim.x) {
      const int g = i % W, r = i / W;
      out[cbase + (long long)r * d.nx + g] = tile[tix(r, g)];
    }
  }
}

// ---------------------------------------------------------------------------
// Z pass with the dyadic Green (or the curl) between forward and inverse FFT.
// MODE_AVG2 : the reference's average of the +s and -s shifted Green functions
//             (s = 1/4 on z).  The pencil psi(z), z < L, is multiplied by
//             exp(-i*pi*z/(2L)), zero-padded to 2L and transformed; bin 2k holds
//             the +s spectrum at k and bin 2k-1 the -s spectrum at k (mod L).
//             After the Green product per bin, the length-2L inverse transform,
//             restricted to z < L and multiplied by exp(+i*pi*z/(2L)), is
//             L*(o_plus + o_minus) up to the constant folded into `scale`.
// MODE_ONE  : one branch with shift sz (0 when z is periodic), ramp table rz.
// MODE_CURL : ik x E with the curl k-index, complex scale folded in.
// ---------------------------------------------------------------------------
enum { ZMODE_AVG2 = 0, ZMODE_ONE = 1, ZMODE_CURL = 2 };

struct GreenParams {
  double dk[3];      // 2*pi/(N_d*res_d) / k_ref
  double shift[3];   // sub-pixel shift of this branch per axis (x, y used in all modes)
  double ksq_re, ksq_im;  // k_square / k_ref^2
  double scale_re, scale_im;  // folded normalisation (and curl factor)
  int curl_index;    // 1 -> curl index formula for odd sizes
  const double* ksq_im_b = nullptr;  // per-RHS imaginary part of k_square (null: ksq_im for all)
  int accumulate = 0;                // 1: add the result to out (second branch of a split average)
};

template <typename R>
__device__ __forceinline__ R kidx_green(int i, int n) {
  const int h = n >> 1;
  return (R)(((i + h) % n) - h);
}
template <typename R>
__device__ __forceinline__ R kidx_curl(int i, int n) {
  return (R)(i < (n >> 1) ? i : i - n);
}

constexpr int ZG_WARPS = 4;  // warps per CTA of the register z pass

// STG (one pencil per warp only): the CTA's warps take x-consecutive pencils at the same (y, b), and the CTA stages
// the 3 x L x W column block in shared memory with coalesced loads and stores (rows of W consecutive x values)
// instead of each lane reading one value per z-plane.  The launcher uses it when nx is a multiple of the warps
// per CTA, so every CTA's warps share (y, b) and leave together.
template <typename S, typename R, int L, int MODE, bool STG = false>
__global__ void __launch_bounds__(256) k_zg(Dims d, const cplx<S>* __restrict__ in, GreenParams gp,
                                            const cplx<R>* __restrict__ twz, const cplx<R>* __restrict__ rz,
                                            cplx<S>* __restrict__ out, const int* __restrict__ active) {
  using T = cplx<R>;
  using TS = cplx<S>;
  constexpr int LF = (MODE == ZMODE_AVG2) ? 2 * L : L;
  using P_ = Plan<LF, R>;
  constexpr int E = P_::E, TP = P_::TP, PW = 32 / TP;
  static_assert(!STG || PW == 1, "the staged z pass takes one pencil per warp");
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tw = reinterpret_cast<T*>(smraw);
  T* twr = tw + LF;
  T* rtab = twr + LF;
  T* ex = rtab + L;
  load_table(tw, twz, 2 * LF);
  if (rz) load_table(rtab, rz, L);
  __syncthreads();
  const int lane = threadIdx.x & 31, wic = threadIdx.x >> 5;
  const int p = lane % PW, t = lane / PW;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + wic;
  const int xg = d.nx / PW;
  const long long total = (long long)xg * d.ny * d.nb;
  if (gw >= total) return;
  const int x = (int)(gw % xg) * PW + p;
  const long long yb = gw / xg;
  const int y = (int)(yb % d.ny);
  const int b = (int)(yb / d.ny);
  if (active && !active[b]) return;
  const long long plane = (long long)d.nx * d.ny;
  const long long base0 = (long long)b * 3 * d.n + (long long)y * d.nx + x;
  T* sm = warp_smem<T, PencilStride<LF, T, TP, false>::v>(ex, wic, PW, p);
  // staged block: row r = (c, z) holds the W pencils' values; the pencil slot is XOR-swizzled with bits 2.. of r,
  // so 16 consecutive rows of one pencil fall in 16 distinct 8-byte bank slots
  constexpr int W = STG ? ZG_WARPS : 1;
  static_assert(!STG || W == 4, "the swizzle assumes 4 pencils per row");
  auto tix = [](int r, int g) { return r * W + (g ^ ((r >> 2) & (W - 1))); };
  TS* tile = reinterpret_cast<TS*>(ex + (size_t)(blockDim.x >> 5) * PW * PencilStride<LF, T, TP, false>::v);
  const long long cbase = base0 - wic;  // the CTA's first pencil (x - wic)
  if constexpr (STG) {
    for (int i = threadIdx.x; i < 3 * L * W; i += blockDim.x) {
      const int g = i % W, r = i / W, c = r / L, z = r - c * L;
      tile[tix(r, g)] = in[cbase + (long long)c * d.n + (long long)z * plane + g];
    }
    __syncthreads();
  }

  T v[3][E];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int z = lay_idx<LF, E, P_::R0>(t, e);
      T a = czero<T>();
      if (MODE != ZMODE_AVG2 || z < L) {
        if constexpr (STG) a = cv<T>(tile[tix(c * L + z, wic)]);
        else a = cv<T>(in[base0 + (long long)c * d.n + (long long)z * plane]);
        if (MODE != ZMODE_CURL && rz) a = cmul(a, rtab[z]);
      }
      v[c][e] = a;
    }
    fft_fwd_plan<-1, P_>(v[c], sm, tw, t);
    __syncwarp();
  }

  // per-bin 3x3 operator
  {
    int kxi = x, kyi = y;
    R kx, ky;
    if (MODE == ZMODE_CURL) {
      kx = (R)gp.dk[0] * kidx_curl<R>(kxi, d.nx);
      ky = (R)gp.dk[1] * kidx_curl<R>(kyi, d.ny);
    } else {
      kx = (R)gp.dk[0] * (kidx_green<R>(kxi, d.nx) + (R)gp.shift[0]);
      ky = (R)gp.dk[1] * (kidx_green<R>(kyi, d.ny) + (R)gp.shift[1]);
    }
    const R ksr = (R)gp.ksq_re, ksi = gp.ksq_im_b ? (R)gp.ksq_im_b[b] : (R)gp.ksq_im;
    const T sc = mk((R)gp.scale_re, (R)gp.scale_im);
    // 1/k_square
    const R kden = ksr * ksr + ksi * ksi;
    const T iks = mk(ksr / kden, -ksi / kden);
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
        // (ik x E) * sc
        T c1 = csub(cscale(e3, ky), cscale(e2, kz));
        T c2 = csub(cscale(e1, kz), cscale(e3, kx));
        T c3 = csub(cscale(e2, kx), cscale(e1, ky));
        const T isc = cmul_i<1>(sc);
        v[0][e] = cmul(c1, isc);
        v[1][e] = cmul(c2, isc);
        v[2][e] = cmul(c3, isc);
      } else {
        T kE = cadd(cadd(cscale(e1, kx), cscale(e2, ky)), cscale(e3, kz));
        kE = cmul(kE, iks);
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
  }

#pragma unroll
  for (int c = 0; c < 3; ++c) {
    fft_rev_plan<+1, P_>(v[c], sm, twr, t);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int z = lay_idx<LF, E, P_::R0>(t, e);
      if (MODE != ZMODE_AVG2 || z < L) {
        T a = v[c][e];
        if (MODE != ZMODE_CURL && rz) a = cmul(a, cconj(rtab[z]));
        if constexpr (STG) {
          tile[tix(c * L + z, wic)] = cv<TS>(a);
        } else {
          const long long o = base0 + (long long)c * d.n + (long long)z * plane;
          if (gp.accumulate) a = cadd(a, cv<T>(out[o]));
          out[o] = cv<TS>(a);
        }
      }
    }
  }
  if constexpr (STG) {
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * L * W; i += blockDim.x) {
      const int g = i % W, r = i / W, c = r / L, z = r - c * L;
      const long long o = cbase + (long long)c * d.n + (long long)z * plane + g;
      TS a = tile[tix(r, g)];
      if (gp.accumulate) {
        const T s2 = cadd(cv<T>(a), cv<T>(out[o]));
        a = cv<TS>(s2);
      }
      out[o] = a;
    }
  }
}

// ---------------------------------------------------------------------------
// XI: inverse FFT along x + epilogue (g += gadd first when given).
//   EPI_STORE    out = g
//   EPI_OP       out = beta*out + alpha*(x - g)                 (CBSLinearOperator)
//   EPI_PREC_OP  out = (i/eps)*V*(xs - g)                       (M^{-1} A x)
//   EPI_PREC_RES out = (i/eps)*V*(bb - xs + g)                  (M^{-1}(b - A x))
// xs = x * rhs_scale[b] when rhs_scale is given.
// ---------------------------------------------------------------------------
enum { EPI_STORE = 0, EPI_OP = 1, EPI_PREC_OP = 2, EPI_PREC_RES = 3 };

struct EpiParams {
  double alpha_re, alpha_im, beta_re, beta_im;
  double inv_eps;  // 1/eps_imag (scaled units)
  const double* inv_eps_b = nullptr;  // per-RHS 1/eps_imag (null: inv_eps for all)
  const double2* shift_b = nullptr;   // EPI_PREC_OP: per-RHS shift theta, out = M^{-1}A x - theta x
  const void* gadd = nullptr;         // storage-typed batch added to g before the epilogue (second branch of a
                                      // two-branch average), element (x, y, z, c, b) at the contiguous batch index
};

// The epilogue on one element: g = G_avg(psi) there, ix its index within RHS b's field, vp its potential value.
template <int EPI, typename S, typename T, typename R>
__device__ __forceinline__ T epi_element(T g, long long ix, const cplx<S>* xvb, const cplx<S>* bvb, const cplx<S>* outb,
                                         const cplx<S>* vp, R ie, R s, T al, T be, const EpiParams& ep, T shf) {
  if constexpr (EPI == EPI_STORE) {
    return g;
  } else if constexpr (EPI == EPI_OP) {
    T xx = cv<T>(xvb[ix]);
    T a = cmul(al, csub(xx, g));
    if (ep.beta_re != 0.0 || ep.beta_im != 0.0) a = cadd(a, cmul(be, cv<T>(outb[ix])));
    return a;
  } else if constexpr (EPI == EPI_PREC_OP) {
    const T vv = cv<T>(*vp);
    const T gam = mk(-vv.y * ie, vv.x * ie);  // (i/eps) * V
    T xx = cscale(cv<T>(xvb[ix]), s);
    T r = cmul(gam, csub(xx, g));
    if (ep.shift_b) r = csub(r, cmul(shf, xx));
    return r;
  } else {
    const T vv = cv<T>(*vp);
    const T gam = mk(-vv.y * ie, vv.x * ie);
    T xx = cscale(cv<T>(xvb[ix]), s);
    return cmul(gam, cadd(csub(cv<T>(bvb[ix]), xx), g));
  }
}

template <typename S, typename R, int L, int EPI>
__global__ void __launch_bounds__(256, (L <= 128 && L != 96) ? 3 : 1) k_xi(Dims d, const cplx<S>* __restrict__ in, const cplx<S>* __restrict__ V,
                                            const cplx<S>* __restrict__ xv, const cplx<S>* __restrict__ bv,
                                            const double* __restrict__ rhs_scale, EpiParams ep,
                                            const cplx<R>* __restrict__ twx, const cplx<R>* __restrict__ rampx,
                                            cplx<S>* __restrict__ out, const int* __restrict__ active, VecTab vt) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int E = P_::E, TP = P_::TP, PW = 32 / TP;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tw = reinterpret_cast<T*>(smraw);
  T* ex = tw + L;
  load_table(tw, twx + L, L);
  __syncthreads();
  const int lane = threadIdx.x & 31, wic = threadIdx.x >> 5;
  const int p = lane / TP, t = lane % TP;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long row = ((long long)blockIdx.x * (blockDim.x >> 5) + wic) * PW + p;
  if (row >= rows) return;
  const int b = (int)(row / ((long long)d.ny * d.nz));
  if (active && !active[b]) return;
  const long long yz = row - (long long)b * d.ny * d.nz;
  T* sm = warp_smem<T, PencilStride<L, T, TP, true>::v>(ex, wic, PW, p);
  // (i/eps) V is formed per component from V (an L1 hit after the first component) rather than held across
  // the three components: the registers it would take decide how many CTAs fit on an SM
  const R ie = (EPI == EPI_PREC_OP || EPI == EPI_PREC_RES) ? (ep.inv_eps_b ? (R)ep.inv_eps_b[b] : (R)ep.inv_eps) : R(0);
  const cplx<S>* Vrow = V + b * d.vstride + yz * L;
  const T shf = (EPI == EPI_PREC_OP && ep.shift_b) ? mk((R)ep.shift_b[b].x, (R)ep.shift_b[b].y) : czero<T>();
  R s = R(1);
  if (rhs_scale) s = (R)rhs_scale[b];
  const T al = mk((R)ep.alpha_re, (R)ep.alpha_im), be = mk((R)ep.beta_re, (R)ep.beta_im);
  const cplx<S>* xvb = vt.in ? (const cplx<S>*)vt.in[b] : xv + (long long)b * 3 * d.n;
  cplx<S>* outb = vt.out ? (cplx<S>*)vt.out[b] : out + (long long)b * 3 * d.n;
  const cplx<S>* bvb = bv + (long long)b * 3 * d.n;
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    const long long base = ((long long)(c + 3 * b) * d.ny * d.nz + yz) * L;
    const long long rbase = ((long long)c * d.ny * d.nz + yz) * L;
    T v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cv<T>(in[base + lay_idx<L, E, P_::RL>(t, e)]);
    fft_rev_plan<+1, P_>(v, sm, tw, t);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = lay_idx<L, E, P_::R0>(t, e);
      const long long ix = rbase + x;
      T g = v[e];
      if (rampx) g = cmul(g, cconj(rampx[x]));
      if (ep.gadd) g = cadd(g, cv<T>(reinterpret_cast<const cplx<S>*>(ep.gadd)[(long long)b * 3 * d.n + ix]));
      const T r = epi_element<EPI, S, T, R>(g, ix, xvb, bvb, outb, Vrow + x, ie, s, al, be, ep, shf);
      outb[ix] = cv<TS>(r);
    }
    __syncwarp();
  }
}

// XI with EPI_PREC_OP followed, on the same rows, by the XF pass (PRO_V) of the next operator application:
//   out  = (i/eps) V (x - g) - theta x          (this application's result, as k_xi stores it)
//   out2 = FFT_x(V .* out)                      (what k_xf would write from the stored out)
// Each row's result is still in registers in the R0 layout that the forward transform takes, so the next
// application's x pass neither reads `out` nor V again.  The forward input is the stored (storage-typed) value,
// so out2 equals k_xf's output bit for bit.  Contiguous batches and no x ramp (the z-only and periodic plans).
template <typename S, typename R, int L>
__global__ void __launch_bounds__(256, (L <= 128 && L != 96) ? 3 : 1) k_xi_xf(Dims d, const cplx<S>* __restrict__ in,
                                                                          const cplx<S>* __restrict__ V,
                                                                          const cplx<S>* __restrict__ xv,
                                                                          EpiParams ep,
                                                                          const cplx<R>* __restrict__ twx,
                                                                          cplx<S>* __restrict__ out,
                                                                          cplx<S>* __restrict__ out2,
                                                                          const int* __restrict__ active) {
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<L, R>;
  constexpr int E = P_::E, TP = P_::TP, PW = 32 / TP;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* twf = reinterpret_cast<T*>(smraw);  // forward-order stage twiddles
  T* twr = twf + L;                      // reversed-order stage twiddles
  T* ex = twr + L;
  load_table(twf, twx, 2 * L);
  __syncthreads();
  const int lane = threadIdx.x & 31, wic = threadIdx.x >> 5;
  const int p = lane / TP, t = lane % TP;
  const long long rows = (long long)d.ny * d.nz * d.nb;
  const long long row = ((long long)blockIdx.x * (blockDim.x >> 5) + wic) * PW + p;
  if (row >= rows) return;  // whole pencils exit together (rows is a multiple of PW)
  const int b = (int)(row / ((long long)d.ny * d.nz));
  if (active && !active[b]) return;
  const long long yz = row - (long long)b * d.ny * d.nz;
  T* sm = warp_smem<T, PencilStride<L, T, TP, true>::v>(ex, wic, PW, p);
  const R ie = ep.inv_eps_b ? (R)ep.inv_eps_b[b] : (R)ep.inv_eps;
  const cplx<S>* Vrow = V + b * d.vstride + yz * L;
  const T shf = ep.shift_b ? mk((R)ep.shift_b[b].x, (R)ep.shift_b[b].y) : czero<T>();
  const T al = mk((R)ep.alpha_re, (R)ep.alpha_im), be = mk((R)ep.beta_re, (R)ep.beta_im);
  const cplx<S>* xvb = xv + (long long)b * 3 * d.n;
  cplx<S>* outb = out + (long long)b * 3 * d.n;
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    const long long base = ((long long)(c + 3 * b) * d.ny * d.nz + yz) * L;
    const long long rbase = ((long long)c * d.ny * d.nz + yz) * L;
    T v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cv<T>(in[base + lay_idx<L, E, P_::RL>(t, e)]);
    fft_rev_plan<+1, P_>(v, sm, twr, t);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = lay_idx<L, E, P_::R0>(t, e);
      const long long ix = rbase + x;
      const T r = epi_element<EPI_PREC_OP, S, T, R>(v[e], ix, xvb, nullptr, outb, Vrow + x, ie, R(1), al, be, ep, shf);
      const TS rs = cv<TS>(r);
      outb[ix] = rs;
      v[e] = cmul(cv<T>(rs), cv<T>(Vrow[x]));  // PRO_V of the next application on the stored value
    }
    __syncwarp();
    fft_fwd_plan<-1, P_>(v, sm, twf, t);
#pragma unroll
    for (int e = 0; e < E; ++e) out2[base + lay_idx<L, E, P_::RL>(t, e)] = cv<TS>(v[e]);
    __syncwarp();
  }
}

}  // namespace fm
