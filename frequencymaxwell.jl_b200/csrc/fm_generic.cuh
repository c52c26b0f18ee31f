// General axis lengths: the Green application and the curl on grids whose padded axes have no fused pass
// (odd lengths, other non-powers of two, e.g. the 201 x 201 x 197 padded grid of the reference's two-beam
// example), and the two sub-pixel-shifted branches on any set of axes.
//
// The work is split into plain passes over the batch, each reading and writing it once:
//   PRE   psi = V.*x [* scale] * ramp_x(x) ramp_y(y) ramp_z(z)       (dyadic_green.jl:243-266, forward ramp)
//   AXIS  1-D DFT along x, y or z (forward exp(-i), or inverse exp(+i) unnormalised), one pencil per lane
//         group as in fm_fft.cuh.  A power-of-two length runs the FFT directly; any other length N runs
//         Bluestein's algorithm (L. Bluestein, "A linear filtering approach to the computation of the discrete
//         Fourier transform", 1970): with c_n = exp(DIR i pi n^2 / N),
//            X_k = c_k * sum_n (x_n c_n) conj(c_{k-n}),
//         a circular convolution evaluated with a power-of-two FFT of length M >= 2N - 1.
//   KSPACE the 3x3 dyadic Green of one branch (dyadic_green.jl:189-221, the Green k index for odd N) or the
//         curl (curl.jl:55-116, the curl k index), with the folded normalisation
//   POST  g = result * conj(ramps) [+ the stored first branch], then the XI epilogue (operator, preconditioner,
//         residual; fm_passes.cuh)
#pragma once
#include "fm_passes.cuh"

namespace fm {

// Tables of one axis for the AXIS pass (arithmetic type R, device pointers).
struct GenAxis {
  int n = 0;                  // axis length
  int m = 0;                  // FFT length: n (a power of two) or the Bluestein length (a power of two >= 2n - 1)
  const void* tw = nullptr;   // [forward-order | reversed-order] stage twiddles of length m (fm_tables.h)
  const void* chirp[2] = {nullptr, nullptr};  // [forward, inverse]: n values c_k = exp(-/+ i pi k^2 / n)
  const void* kern[2] = {nullptr, nullptr};   // [forward, inverse]: m values FFT_m(conj(c) wrapped) / m
};

struct GenRamps {
  const void* r[3] = {nullptr, nullptr, nullptr};  // per-axis forward ramps of this branch (null: unshifted)
};

// AXIS: DIR = -1 forward DFT, +1 inverse (unnormalised), along `axis` of a batch of 3-component fields.  A lane
// group reads its whole pencil before it writes, and pencils do not overlap, so the pass may run in place.
template <typename S, typename R, int M, int DIR>
__global__ void __launch_bounds__(256) k_gen_axis(Dims d, int axis, const cplx<S>* in, cplx<S>* out, GenAxis ax,
                                                  const int* __restrict__ active) {  // in may equal out
  using T = cplx<R>;
  using TS = cplx<S>;
  using P_ = Plan<M, R>;
  constexpr int E = P_::E, TP = P_::TP, PW = 32 / TP;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* tw = reinterpret_cast<T*>(smraw);
  T* twr = tw + M;
  T* ex = twr + M;
  load_table(tw, (const T*)ax.tw, 2 * M);
  __syncthreads();
  const int lane = threadIdx.x & 31, wic = threadIdx.x >> 5;
  const int p = lane / TP, t = lane % TP;
  const int N = ax.n;
  const long long plane = (long long)d.nx * d.ny;
  const long long pencils = d.n / N * 3 * d.nb;
  const long long pen = ((long long)blockIdx.x * (blockDim.x >> 5) + wic) * PW + p;
  const bool on = pen < pencils;
  long long base = 0, stride = 1;
  if (on) {
    if (axis == 0) {
      base = pen * d.nx;
    } else if (axis == 1) {
      const long long x = pen % d.nx, r = pen / d.nx;  // r = z + nz*(c + 3b)
      base = x + r * plane;
      stride = d.nx;
    } else {
      const long long xy = pen % plane, cb = pen / plane;
      base = xy + cb * d.n;
      stride = plane;
    }
  }
  const int b = on ? (int)(base / (3 * d.n)) : 0;
  const bool live = on && !(active && !active[b]);
  T* sm = warp_smem<T, PencilStride<M, T, TP, true>::v>(ex, wic, PW, p);
  const bool blue = N != M;
  const T* ch = blue ? (const T*)ax.chirp[DIR < 0 ? 0 : 1] : nullptr;
  T v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = lay_idx<M, E, P_::R0>(t, e);
    T a = czero<T>();
    if (live && i < N) {
      a = cv<T>(in[base + (long long)i * stride]);
      if (blue) a = cmul(a, ch[i]);
    }
    v[e] = a;
  }
  if (!blue) {
    fft_fwd_plan<DIR, P_>(v, sm, tw, t);
    if (live) {
#pragma unroll
      for (int e = 0; e < E; ++e) out[base + (long long)lay_idx<M, E, P_::RL>(t, e) * stride] = cv<TS>(v[e]);
    }
    return;
  }
  fft_fwd_plan<-1, P_>(v, sm, tw, t);
  const T* kk = (const T*)ax.kern[DIR < 0 ? 0 : 1];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = cmul(v[e], kk[lay_idx<M, E, P_::RL>(t, e)]);
  __syncwarp();
  fft_rev_plan<+1, P_>(v, sm, twr, t);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int k = lay_idx<M, E, P_::R0>(t, e);
      if (k < N) out[base + (long long)k * stride] = cv<TS>(cmul(v[e], ch[k]));
    }
  }
}

// element i of the batch -> (x, y, z, c, b) parts
struct GenIdx {
  int x, y, z, b;
  long long xyz, ix;  // voxel index, index within RHS b's field
};
__device__ __forceinline__ GenIdx gen_idx(const Dims& d, long long i) {
  GenIdx g;
  const long long f = 3 * d.n;
  g.b = (int)(i / f);
  g.ix = i - (long long)g.b * f;
  g.xyz = g.ix % d.n;
  g.x = (int)(g.xyz % d.nx);
  const long long r = g.xyz / d.nx;
  g.y = (int)(r % d.ny);
  g.z = (int)(r / d.ny);
  return g;
}

template <typename R>
__device__ __forceinline__ cplx<R> ramp3(const GenRamps& rp, const GenIdx& g) {
  using T = cplx<R>;
  T w = mk(R(1), R(0));
  if (rp.r[0]) w = cmul(w, ((const T*)rp.r[0])[g.x]);
  if (rp.r[1]) w = cmul(w, ((const T*)rp.r[1])[g.y]);
  if (rp.r[2]) w = cmul(w, ((const T*)rp.r[2])[g.z]);
  return w;
}

// PRE: out = in [.* V [* rs[b]]] * ramps  (PRO_COPY / PRO_V / PRO_V_SCALE as in k_xf)
template <typename S, typename R, int PRO>
__global__ void __launch_bounds__(256) k_gen_pre(Dims d, const cplx<S>* __restrict__ in, const cplx<S>* __restrict__ V,
                                                 const double* __restrict__ rhs_scale, GenRamps rp,
                                                 cplx<S>* __restrict__ out, const int* __restrict__ active, VecTab vt) {
  using T = cplx<R>;
  const long long total = 3 * d.n * d.nb;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const GenIdx g = gen_idx(d, i);
    if (active && !active[g.b]) continue;
    const cplx<S>* inb = vt.in ? (const cplx<S>*)vt.in[g.b] : in + (long long)g.b * 3 * d.n;
    T a = cv<T>(inb[g.ix]);
    if constexpr (PRO != PRO_COPY) a = cmul(a, cv<T>(V[g.b * d.vstride + g.xyz]));
    if constexpr (PRO == PRO_V_SCALE) a = cscale(a, (R)rhs_scale[g.b]);
    a = cmul(a, ramp3<R>(rp, g));
    out[i] = cv<cplx<S>>(a);
  }
}

// KSPACE: in place.  ZMODE_ONE: the Green of one branch (shifts in gp.shift); ZMODE_CURL: i k x E.
// Both scaled by gp.scale.
template <typename S, typename R, int MODE>
__global__ void __launch_bounds__(256) k_gen_kspace(Dims d, cplx<S>* __restrict__ f, GreenParams gp,
                                                    const int* __restrict__ active) {
  using T = cplx<R>;
  const long long total = d.n * d.nb;
  const T sc = mk((R)gp.scale_re, (R)gp.scale_im);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / d.n);
    if (active && !active[b]) continue;
    const long long xyz = i - (long long)b * d.n;
    const int x = (int)(xyz % d.nx);
    const long long r = xyz / d.nx;
    const int y = (int)(r % d.ny), z = (int)(r / d.ny);
    cplx<S>* fb = f + (long long)b * 3 * d.n + xyz;
    const T e1 = cv<T>(fb[0]), e2 = cv<T>(fb[d.n]), e3 = cv<T>(fb[2 * d.n]);
    T o1, o2, o3;
    if constexpr (MODE == ZMODE_CURL) {
      const R kx = (R)gp.dk[0] * kidx_curl<R>(x, d.nx), ky = (R)gp.dk[1] * kidx_curl<R>(y, d.ny),
              kz = (R)gp.dk[2] * kidx_curl<R>(z, d.nz);
      const T isc = cmul_i<1>(sc);
      o1 = cmul(csub(cscale(e3, ky), cscale(e2, kz)), isc);
      o2 = cmul(csub(cscale(e1, kz), cscale(e3, kx)), isc);
      o3 = cmul(csub(cscale(e2, kx), cscale(e1, ky)), isc);
    } else {
      const R kx = (R)gp.dk[0] * (kidx_green<R>(x, d.nx) + (R)gp.shift[0]);
      const R ky = (R)gp.dk[1] * (kidx_green<R>(y, d.ny) + (R)gp.shift[1]);
      const R kz = (R)gp.dk[2] * (kidx_green<R>(z, d.nz) + (R)gp.shift[2]);
      const R ksr = (R)gp.ksq_re, ksi = gp.ksq_im_b ? (R)gp.ksq_im_b[b] : (R)gp.ksq_im;
      const R kden = ksr * ksr + ksi * ksi;
      const T iks = mk(ksr / kden, -ksi / kden);
      const T kE = cmul(cadd(cadd(cscale(e1, kx), cscale(e2, ky)), cscale(e3, kz)), iks);
      const R dr = kx * kx + ky * ky + kz * kz - ksr, di = -ksi;
      const R rdd = R(1) / (dr * dr + di * di);
      const T fac = cmul(sc, mk(dr * rdd, -di * rdd));
      o1 = cmul(csub(e1, cscale(kE, kx)), fac);
      o2 = cmul(csub(e2, cscale(kE, ky)), fac);
      o3 = cmul(csub(e3, cscale(kE, kz)), fac);
    }
    fb[0] = cv<cplx<S>>(o1);
    fb[d.n] = cv<cplx<S>>(o2);
    fb[2 * d.n] = cv<cplx<S>>(o3);
  }
}

// POST: g = in * conj(ramps) [+ ep.gadd], then the epilogue EPI (fm_passes.cuh, epi_element) into out.
template <typename S, typename R, int EPI>
__global__ void __launch_bounds__(256) k_gen_post(Dims d, const cplx<S>* __restrict__ in, const cplx<S>* __restrict__ V,
                                                  const cplx<S>* __restrict__ xv, const cplx<S>* __restrict__ bv,
                                                  const double* __restrict__ rhs_scale, EpiParams ep, GenRamps rp,
                                                  cplx<S>* __restrict__ out, const int* __restrict__ active, VecTab vt) {
  using T = cplx<R>;
  const long long total = 3 * d.n * d.nb;
  const T al = mk((R)ep.alpha_re, (R)ep.alpha_im), be = mk((R)ep.beta_re, (R)ep.beta_im);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const GenIdx g = gen_idx(d, i);
    const int b = g.b;
    if (active && !active[b]) continue;
    T gv = cmul(cv<T>(in[i]), cconj(ramp3<R>(rp, g)));
    if (ep.gadd) gv = cadd(gv, cv<T>(reinterpret_cast<const cplx<S>*>(ep.gadd)[i]));
    const R ie = (EPI == EPI_PREC_OP || EPI == EPI_PREC_RES) ? (ep.inv_eps_b ? (R)ep.inv_eps_b[b] : (R)ep.inv_eps) : R(0);
    const T shf = (EPI == EPI_PREC_OP && ep.shift_b) ? mk((R)ep.shift_b[b].x, (R)ep.shift_b[b].y) : czero<T>();
    const R s = rhs_scale ? (R)rhs_scale[b] : R(1);
    const cplx<S>* xvb = vt.in ? (const cplx<S>*)vt.in[b] : xv + (long long)b * 3 * d.n;
    cplx<S>* outb = vt.out ? (cplx<S>*)vt.out[b] : out + (long long)b * 3 * d.n;
    const cplx<S>* bvb = bv + (long long)b * 3 * d.n;
    const T r = epi_element<EPI, S, T, R>(gv, g.ix, xvb, bvb, outb, V + b * d.vstride + g.xyz, ie, s, al, be, ep, shf);
    outb[g.ix] = cv<cplx<S>>(r);
  }
}

}  // namespace fm
