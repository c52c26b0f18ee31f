// Batched Krylov vector kernels with FP64 accumulation.
//
// A batch holds B right-hand sides; each vector of one RHS has M complex
// entries (M = 3 * padded voxels).  A family of K basis vectors is stored as
// U[(i*B + b)*M + e].  Reductions are deterministic: each block writes its
// partial sums, and the last block of an RHS (ticket counter) adds the
// partials in block order.
#pragma once
#include "fm_complex.cuh"

namespace fm {

constexpr int KV_THREADS = 256;
constexpr int KV_WARPS = KV_THREADS / 32;
constexpr int KV_EPT = 8;          // elements per thread per chunk
constexpr int KV_KMAX = 128;       // max vectors in one multi-dot / update

__device__ __forceinline__ double2 warp_sum(double2 a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a.x += __shfl_xor_sync(0xffffffffu, a.x, o);
    a.y += __shfl_xor_sync(0xffffffffu, a.y, o);
  }
  return a;
}

// Reduction tail shared by the kernels below.  Each block has written
// part[(b*nblk + blk)*K + i]; the last block of RHS b writes out[b*K + i].
__device__ __forceinline__ void finish_reduce(double2* part, double2* out, unsigned* counter, int K, int nblk,
                                              int b) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned tk = atomicAdd(&counter[b], 1u);
    last = (tk == (unsigned)(nblk - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int i = threadIdx.x; i < K; i += blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    for (int k = 0; k < nblk; ++k) {
      double2 v = __ldcg(&part[((size_t)b * nblk + k) * K + i]);
      s.x += v.x;
      s.y += v.y;
    }
    out[(size_t)b * K + i] = s;
  }
  if (threadIdx.x == 0) counter[b] = 0;
}

// out[b][i] = sum_e conj(U_i[b][e]) * w[b][e]   (i < K), plus out[b][K] = ||w||^2 when WNORM.
// Optional per-RHS arguments: wtab[b] replaces w + b*M, Kb[b] (<= K) the number of basis vectors.
template <typename R, bool WNORM>
__global__ void __launch_bounds__(KV_THREADS) k_multidot(long long M, int B, int K, const cplx<R>* __restrict__ U,
                                                         const cplx<R>* __restrict__ w, double2* __restrict__ part,
                                                         double2* __restrict__ out, unsigned* __restrict__ counter,
                                                         const int* __restrict__ active,
                                                         const cplx<R>* const* __restrict__ wtab = nullptr,
                                                         const int* __restrict__ Kb = nullptr) {
  using T = cplx<R>;
  __shared__ double2 acc[KV_WARPS][KV_KMAX + 1];
  const int b = blockIdx.y, nblk = gridDim.x;
  const int KK = K + (WNORM ? 1 : 0);
  if (active && !active[b]) return;  // uniform per block; no reduction is issued for inactive RHS
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  for (int i = lane; i < KK; i += 32) acc[wi][i] = make_double2(0.0, 0.0);
  __syncwarp();
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long per = ((M + nblk - 1) / nblk + chunk - 1) / chunk * chunk;
  const long long lo = (long long)blockIdx.x * per, hi = min(M, lo + per);
  const T* wb = wtab ? wtab[b] : w + (size_t)b * M;
  const int Kr = Kb ? Kb[b] : K;
  for (long long c0 = lo; c0 < hi; c0 += chunk) {
    double2 wv[KV_EPT];
#pragma unroll
    for (int k = 0; k < KV_EPT; ++k) {
      long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
      wv[k] = e < hi ? to_d(wb[e]) : make_double2(0.0, 0.0);
    }
    for (int i = 0; i < Kr; ++i) {
      const T* ub = U + ((size_t)i * B + b) * M;
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < KV_EPT; ++k) {
        long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
        if (e < hi) {
          double2 u = to_d(ub[e]);
          s.x = fma(u.x, wv[k].x, fma(u.y, wv[k].y, s.x));
          s.y = fma(u.x, wv[k].y, fma(-u.y, wv[k].x, s.y));
        }
      }
      s = warp_sum(s);
      if (lane == 0) { acc[wi][i].x += s.x; acc[wi][i].y += s.y; }
    }
    if constexpr (WNORM) {
      double2 s = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < KV_EPT; ++k) s.x = fma(wv[k].x, wv[k].x, fma(wv[k].y, wv[k].y, s.x));
      s = warp_sum(s);
      if (lane == 0) acc[wi][K].x += s.x;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < KK; i += blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    for (int q = 0; q < KV_WARPS; ++q) { s.x += acc[q][i].x; s.y += acc[q][i].y; }
    part[((size_t)b * nblk + blockIdx.x) * KK + i] = s;
  }
  finish_reduce(part, out, counter, KK, nblk, b);
}

// Coefficient source for the update kernels.  For RHS b and vector i the
// coefficient is  sgn * h[b*hs + i] * sc[i*ss + b]^2  (sc = deferred basis
// normalisation, 1 when null; the square because both the projection and the
// subtracted vector carry the scale).  With POW1 the scale enters once.
struct Coef {
  const double2* h;
  int hs;
  const double* sc;
  int ss;
  double sgn;
  int pow1;
  __device__ __forceinline__ double2 get(int b, int i) const {
    double2 c = h[(size_t)b * hs + i];
    double f = sgn;
    if (sc) {
      double s = sc[(size_t)i * ss + b];
      f *= pow1 ? s : s * s;
    }
    return make_double2(c.x * f, c.y * f);
  }
};

// w[b] = a0[b]*w[b] + sum_i coef(b,i) * U_i[b]   (FP64 accumulation); optional ||w'||^2.
// a0 scale (real) is taken from w_scale[b] when given, else 1.
template <typename R, bool NORM>
__global__ void __launch_bounds__(KV_THREADS) k_update(long long M, int B, int K, const cplx<R>* __restrict__ U,
                                                       Coef cf, cplx<R>* __restrict__ w, const double* __restrict__ w_scale,
                                                       double2* __restrict__ part, double2* __restrict__ out,
                                                       unsigned* __restrict__ counter, const int* __restrict__ active,
                                                       cplx<R>* const* __restrict__ wtab = nullptr,
                                                       const int* __restrict__ Kb = nullptr) {
  using T = cplx<R>;
  __shared__ double2 cs[KV_KMAX];
  __shared__ double red[KV_WARPS];
  const int b = blockIdx.y, nblk = gridDim.x;
  if (active && !active[b]) return;
  const int Kr = Kb ? Kb[b] : K;
  for (int i = threadIdx.x; i < Kr; i += blockDim.x) cs[i] = cf.get(b, i);
  __syncthreads();
  const double a0 = w_scale ? w_scale[b] : 1.0;
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long per = ((M + nblk - 1) / nblk + chunk - 1) / chunk * chunk;
  const long long lo = (long long)blockIdx.x * per, hi = min(M, lo + per);
  T* wb = wtab ? wtab[b] : w + (size_t)b * M;
  double nrm = 0.0;
  for (long long c0 = lo; c0 < hi; c0 += chunk) {
    double2 acc[KV_EPT];
#pragma unroll
    for (int k = 0; k < KV_EPT; ++k) {
      long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
      double2 v = e < hi ? to_d(wb[e]) : make_double2(0.0, 0.0);
      acc[k] = make_double2(v.x * a0, v.y * a0);
    }
    for (int i = 0; i < Kr; ++i) {
      const T* ub = U + ((size_t)i * B + b) * M;
      const double2 c = cs[i];
#pragma unroll
      for (int k = 0; k < KV_EPT; ++k) {
        long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
        if (e < hi) {
          double2 u = to_d(ub[e]);
          acc[k].x = fma(c.x, u.x, fma(-c.y, u.y, acc[k].x));
          acc[k].y = fma(c.x, u.y, fma(c.y, u.x, acc[k].y));
        }
      }
    }
#pragma unroll
    for (int k = 0; k < KV_EPT; ++k) {
      long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
      if (e < hi) {
        T r = from_d<T>(acc[k]);
        wb[e] = r;
        if constexpr (NORM) {
          double2 rd = to_d(r);
          nrm = fma(rd.x, rd.x, fma(rd.y, rd.y, nrm));
        }
      }
    }
  }
  if constexpr (NORM) {
    double2 s = warp_sum(make_double2(nrm, 0.0));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s.x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < KV_WARPS; ++q) t += red[q];
      part[(size_t)b * nblk + blockIdx.x] = make_double2(t, 0.0);
    }
    finish_reduce(part, out, counter, 1, nblk, b);
  }
}

// One step of modified Gram-Schmidt as Krylov.jl runs it (sc[i*ss + b] scales U_i):
//   if i > 0:  w -= h_{i-1} * v_{i-1}        (h read from device, v = sc*U)
//   if i < K:  h_i = <v_i, w>                (reduced into hout[b*hs + i])
//   else:      hout[b*hs + K] = ||w||^2
template <typename R>
__global__ void __launch_bounds__(KV_THREADS) k_mgs(long long M, int B, int i, int K, const cplx<R>* __restrict__ U,
                                                    const double* __restrict__ sc, int ss, cplx<R>* __restrict__ w,
                                                    double2* __restrict__ hout, int hs, double2* __restrict__ part,
                                                    unsigned* __restrict__ counter, const int* __restrict__ active) {
  using T = cplx<R>;
  __shared__ double2 red[KV_WARPS];
  const int b = blockIdx.y, nblk = gridDim.x;
  if (active && !active[b]) return;
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long per = ((M + nblk - 1) / nblk + chunk - 1) / chunk * chunk;
  const long long lo = (long long)blockIdx.x * per, hi = min(M, lo + per);
  T* wb = w + (size_t)b * M;
  double2 cprev = make_double2(0.0, 0.0);
  const T* up = nullptr;
  if (i > 0) {
    double2 h = hout[(size_t)b * hs + (i - 1)];
    double s = sc ? sc[(size_t)(i - 1) * ss + b] : 1.0;
    cprev = make_double2(-h.x * s, -h.y * s);
    up = U + ((size_t)(i - 1) * B + b) * M;
  }
  const T* ui = (i < K) ? U + ((size_t)i * B + b) * M : nullptr;
  const double si = (i < K && sc) ? sc[(size_t)i * ss + b] : 1.0;
  double2 acc = make_double2(0.0, 0.0);
  for (long long c0 = lo; c0 < hi; c0 += chunk) {
#pragma unroll
    for (int k = 0; k < KV_EPT; ++k) {
      long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
      if (e < hi) {
        double2 wv = to_d(wb[e]);
        if (up) {
          double2 u = to_d(up[e]);
          wv.x = fma(cprev.x, u.x, fma(-cprev.y, u.y, wv.x));
          wv.y = fma(cprev.x, u.y, fma(cprev.y, u.x, wv.y));
          T r = from_d<T>(wv);
          wb[e] = r;
          wv = to_d(r);
        }
        if (ui) {
          double2 u = to_d(ui[e]);
          acc.x = fma(u.x, wv.x, fma(u.y, wv.y, acc.x));
          acc.y = fma(u.x, wv.y, fma(-u.y, wv.x, acc.y));
        } else {
          acc.x = fma(wv.x, wv.x, fma(wv.y, wv.y, acc.x));
        }
      }
    }
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < KV_WARPS; ++q) { t.x += red[q].x; t.y += red[q].y; }
    if (ui) { t.x *= si; t.y *= si; }
    part[(size_t)b * nblk + blockIdx.x] = t;
  }
  // reduce into hout[b*hs + i]
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&counter[b], 1u) == (unsigned)(nblk - 1));
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double2 s = make_double2(0.0, 0.0);
    for (int k = 0; k < nblk; ++k) {
      double2 v = __ldcg(&part[(size_t)b * nblk + k]);
      s.x += v.x;
      s.y += v.y;
    }
    hout[(size_t)b * hs + i] = s;
    counter[b] = 0;
  }
}

// Generic batched elementwise combination (FP64 arithmetic):
//   y[b] = ca[b]*a[b] + cb[b]*bv[b] + cc[b]*c[b]     (missing operands are skipped)
// coefficients are complex per RHS.  Optionally reduces ||y||^2 into out[b].
template <typename R, bool NORM>
__global__ void __launch_bounds__(KV_THREADS) k_axpby3(long long M, const cplx<R>* __restrict__ a, const double2* __restrict__ ca,
                                                       const cplx<R>* __restrict__ bv, const double2* __restrict__ cb,
                                                       const cplx<R>* __restrict__ c, const double2* __restrict__ cc,
                                                       cplx<R>* __restrict__ y, double2* __restrict__ part,
                                                       double2* __restrict__ out, unsigned* __restrict__ counter,
                                                       const int* __restrict__ active) {
  using T = cplx<R>;
  __shared__ double red[KV_WARPS];
  const int b = blockIdx.y, nblk = gridDim.x;
  if (active && !active[b]) return;
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long per = ((M + nblk - 1) / nblk + chunk - 1) / chunk * chunk;
  const long long lo = (long long)blockIdx.x * per, hi = min(M, lo + per);
  const size_t off = (size_t)b * M;
  const double2 A = ca ? ca[b] : make_double2(0, 0), Bc = cb ? cb[b] : make_double2(0, 0),
                C = cc ? cc[b] : make_double2(0, 0);
  double nrm = 0.0;
  for (long long c0 = lo; c0 < hi; c0 += chunk) {
#pragma unroll
    for (int k = 0; k < KV_EPT; ++k) {
      long long e = c0 + (long long)k * KV_THREADS + threadIdx.x;
      if (e < hi) {
        double2 r = make_double2(0.0, 0.0);
        if (a) { double2 u = to_d(a[off + e]); r.x = fma(A.x, u.x, fma(-A.y, u.y, r.x)); r.y = fma(A.x, u.y, fma(A.y, u.x, r.y)); }
        if (bv) { double2 u = to_d(bv[off + e]); r.x = fma(Bc.x, u.x, fma(-Bc.y, u.y, r.x)); r.y = fma(Bc.x, u.y, fma(Bc.y, u.x, r.y)); }
        if (c) { double2 u = to_d(c[off + e]); r.x = fma(C.x, u.x, fma(-C.y, u.y, r.x)); r.y = fma(C.x, u.y, fma(C.y, u.x, r.y)); }
        T o = from_d<T>(r);
        y[off + e] = o;
        if constexpr (NORM) { double2 od = to_d(o); nrm = fma(od.x, od.x, fma(od.y, od.y, nrm)); }
      }
    }
  }
  if constexpr (NORM) {
    double2 s = warp_sum(make_double2(nrm, 0.0));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s.x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int q = 0; q < KV_WARPS; ++q) t += red[q];
      part[(size_t)b * nblk + blockIdx.x] = make_double2(t, 0.0);
    }
    finish_reduce(part, out, counter, 1, nblk, b);
  }
}

}  // namespace fm
