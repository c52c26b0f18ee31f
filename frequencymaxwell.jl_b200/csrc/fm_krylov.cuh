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

// ---------------------------------------------------------------------------
// Block (s-step) Gram-Schmidt kernels.  The basis of RHS b is the sequence of
// stored vectors X_k = U[(k*B + b)*M], k < K; the S block vectors are
// Y_t = Y[(t*B + b)*M] in their own buffer and type TY (complex FP64 or the
// basis type).  M must be a multiple of 4.
// ---------------------------------------------------------------------------

// out[b] = sum_{a<n} c[b*cs + a] * X_{k0+a}[b]   (FP64 accumulation; n <= 16).  Optional per-RHS k0b[b], nb[b]
// replace k0 and n.
template <typename R, typename TY>
__global__ void __launch_bounds__(KV_THREADS) k_combine(long long M, int B, int k0, int n, const cplx<R>* __restrict__ U,
                                                        const double2* __restrict__ c, int cs, TY* __restrict__ out,
                                                        const int* __restrict__ active,
                                                        const int* __restrict__ k0b = nullptr,
                                                        const int* __restrict__ nb = nullptr) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  if (k0b) k0 = k0b[b];
  if (nb) n = nb[b];
  __shared__ double2 cc[16];
  if (threadIdx.x < n) cc[threadIdx.x] = c[(size_t)b * cs + threadIdx.x];
  __syncthreads();
  TY* ob = out + (size_t)b * M;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < M; e += (long long)gridDim.x * blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int a = 0; a < n; ++a) {
      const double2 x = to_d(U[((size_t)(k0 + a) * B + b) * M + e]);
      acc.x = fma(cc[a].x, x.x, fma(-cc[a].y, x.y, acc.x));
      acc.y = fma(cc[a].x, x.y, fma(cc[a].y, x.x, acc.y));
    }
    ob[e] = from_d<TY>(acc);
  }
}
// ---------------------------------------------------------------------------
// FP64 tensor-core (mma.sync m8n8k4 .f64) forms of the block dot and block
// update.  For S <= 4 the real and imaginary parts of the S block vectors (or
// coefficients) fill the 8 columns of the B operand (columns t: real part of
// vector t, 4 + t: imaginary part; columns of t >= S are zero); for S <= 8 two
// B tiles hold the real and the imaginary parts.  The real and imaginary parts of
// the basis values are the A operands of two MMAs per tile, P and Q, so that for
// column t (one tile)
//   conj(x) y:  Re = P[t] + Q[4+t],   Im = P[4+t] - Q[t]
//   x c:        Re = P[t] - Q[4+t],   Im = P[4+t] + Q[t].
// Fragment layout of m8n8k4 (row.col): A[gid][tig], B[tig][gid] and
// C[gid][2 tig + i] for lane = 4 gid + tig.  Each lane reads a run of four
// consecutive elements (32 bytes of complex FP32); the summed element index is
// permuted in the same way for both operands, which leaves the products as they are.
// ---------------------------------------------------------------------------
// four consecutive complex values starting at a 32-byte aligned address (two or four 128-bit loads)
__device__ __forceinline__ void load4(const float2* p, float2 (&v)[4]) {
  const float4 a = reinterpret_cast<const float4*>(p)[0], c = reinterpret_cast<const float4*>(p)[1];
  v[0] = make_float2(a.x, a.y);
  v[1] = make_float2(a.z, a.w);
  v[2] = make_float2(c.x, c.y);
  v[3] = make_float2(c.z, c.w);
}
__device__ __forceinline__ void load4(const double2* p, double2 (&v)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = p[q];
}

// (not volatile: the MMA has no effect beyond its outputs, so the scheduler may move loads across it)
__device__ __forceinline__ void mma_f64(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// D[b][k*S + t] = sum_e conj(X_k[e]) * Y_t[e]   (FP64 tensor cores, deterministic; S <= 16).  Optional per-RHS
// basis sizes Kb[b] <= K: the rows k >= Kb[b] of RHS b come out zero (the output keeps the stride K*S).
// S <= 4: one B tile; S > 4: NTH = ceil(S/8) tiles of real parts then NTH tiles of imaginary parts (tile h holds
// block vectors 8h .. 8h+7 in its columns), so that for t = 8h + c
//   Re = P[h][c] + Q[NTH + h][c],  Im = P[NTH + h][c] - Q[h][c]  within each lane.
// WIDE (5 <= S <= 8): four groups of 8 basis vectors per warp and one run of 4 elements per lane in a warp step,
// instead of two groups and two runs: the same MMAs per step from a quarter fewer loaded bytes, and half the
// re-reads of the block vectors across the warps along the basis.
template <typename R, typename TY, int S, bool WIDE = false>
__global__ void __launch_bounds__(KV_THREADS, (S > 8 || WIDE) ? 2 : 1) k_blockdot_mma(long long M, int B, int K, const cplx<R>* __restrict__ U,
                                                             const TY* __restrict__ Y, double2* __restrict__ part,
                                                             double2* __restrict__ out, unsigned* __restrict__ counter,
                                                             const int* __restrict__ active,
                                                             const int* __restrict__ Kb = nullptr) {
  static_assert(S >= 1 && S <= 16, "block dot on tensor cores takes 1..16 block vectors");
  static_assert(!WIDE || (S > 4 && S <= 8), "the wide form is for 5..8 block vectors");
  using T = cplx<R>;
  constexpr int NTH = S <= 4 ? 1 : (S + 7) / 8;  // 8-column tiles per part
  constexpr int NT = S <= 4 ? 1 : 2 * NTH;       // B tiles
  constexpr int GPW = (S <= 4 || WIDE) ? 4 : 2;  // groups of 8 basis vectors per warp
  constexpr int HR = (S <= 8 && !WIDE) ? 2 : 1;  // runs of 4 elements per lane in a warp step
  constexpr int WSTEP = 16 * HR;                 // elements per warp step
  __shared__ double2 red[KV_WARPS][GPW * 8][S];
  const int b = blockIdx.y, nblk = gridDim.x;
  if (active && !active[b]) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  // KW warps along the basis (GPW groups of 8 vectors each) x EW along the elements; the launcher sizes the CTA
  // as 32 * KW * EW threads (at most KV_THREADS) so that no warp idles
  const int KG = (K + 7) >> 3, KW = (KG + GPW - 1) / GPW, EW = (int)(blockDim.x >> 5) / KW;
  const int kw = w % KW, ew = w / KW;
  const int Kr = Kb ? Kb[b] : K;  // basis vectors of this RHS
  double P[GPW][NT][2], Q[GPW][NT][2];
#pragma unroll
  for (int g = 0; g < GPW; ++g)
#pragma unroll
    for (int n = 0; n < NT; ++n) P[g][n][0] = P[g][n][1] = Q[g][n][0] = Q[g][n][1] = 0.0;
  const long long per = ((M + nblk - 1) / nblk + 31) / 32 * 32;
  const long long lo = (long long)blockIdx.x * per, hi = min(M, lo + per);
  const size_t us = (size_t)B * M;
  const T* ub = U + (size_t)b * M;
  const TY* yb = Y + (size_t)b * M;
  if (ew < EW) {
    // a warp step covers WSTEP elements: HR runs of 4 per lane
    for (long long e0 = lo + (long long)ew * WSTEP; e0 < hi; e0 += (long long)EW * WSTEP) {
      double bf[NT][HR][4];
      bool ein[HR];
#pragma unroll
      for (int h = 0; h < HR; ++h) {
        const long long eb = e0 + 16 * h + 4 * tig;  // wholly inside or outside the range
        ein[h] = eb < hi;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if constexpr (NT == 1) {
            const int yt = gid & 3;  // block vector of this lane's B column
            double2 y = make_double2(0.0, 0.0);
            if (yt < S && ein[h]) y = to_d(yb[yt * us + eb + q]);
            bf[0][h][q] = gid >= 4 ? y.y : y.x;
          } else {
#pragma unroll
            for (int th = 0; th < NTH; ++th) {
              const int yt = 8 * th + gid;
              double2 y = make_double2(0.0, 0.0);
              if (yt < S && ein[h]) y = to_d(yb[yt * us + eb + q]);
              bf[th][h][q] = y.x;
              bf[NTH + th][h][q] = y.y;
            }
          }
        }
      }
#pragma unroll
      for (int g = 0; g < GPW; ++g) {
        if ((kw * GPW + g) * 8 >= Kr) break;  // warp-uniform
        const int k = (kw * GPW + g) * 8 + gid;
        T xv[HR][4];
#pragma unroll
        for (int h = 0; h < HR; ++h) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            xv[h][q].x = 0;
            xv[h][q].y = 0;
          }
          if (k < Kr && ein[h]) load4(ub + (size_t)k * us + e0 + 16 * h + 4 * tig, xv[h]);
        }
#pragma unroll
        for (int h = 0; h < HR; ++h)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double2 x = to_d(xv[h][q]);
#pragma unroll
            for (int n = 0; n < NT; ++n) {
              mma_f64(P[g][n][0], P[g][n][1], x.x, bf[n][h][q]);
              mma_f64(Q[g][n][0], Q[g][n][1], x.y, bf[n][h][q]);
            }
          }
      }
    }
  }
#pragma unroll
  for (int g = 0; g < GPW; ++g) {
    if constexpr (NT == 1) {
      // columns 2 tig, 2 tig + 1 of P and Q; the partner lane tig ^ 2 holds columns 4 + (2 tig, 2 tig + 1)
      const double pp0 = __shfl_xor_sync(0xffffffffu, P[g][0][0], 2), pp1 = __shfl_xor_sync(0xffffffffu, P[g][0][1], 2);
      const double qp0 = __shfl_xor_sync(0xffffffffu, Q[g][0][0], 2), qp1 = __shfl_xor_sync(0xffffffffu, Q[g][0][1], 2);
      if (tig < 2) {
        const int t0 = 2 * tig;
        if (t0 < S) red[w][g * 8 + gid][t0] = make_double2(P[g][0][0] + qp0, pp0 - Q[g][0][0]);
        if (t0 + 1 < S) red[w][g * 8 + gid][t0 + 1] = make_double2(P[g][0][1] + qp1, pp1 - Q[g][0][1]);
      }
    } else {
#pragma unroll
      for (int th = 0; th < NTH; ++th)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int t = 8 * th + 2 * tig + i;
          if (t < S)
            red[w][g * 8 + gid][t] =
                make_double2(P[g][th][i] + Q[g][NTH + th][i], P[g][NTH + th][i] - Q[g][th][i]);
        }
    }
  }
  __syncthreads();
  const int KS = K * S;
  for (int o = threadIdx.x; o < KS; o += blockDim.x) {
    const int k = o / S, t = o - k * S;
    const int kg = k >> 3, kwo = kg / GPW, g = kg - kwo * GPW;
    double2 sum = make_double2(0.0, 0.0);
    for (int e = 0; e < EW; ++e) {
      const double2 v = red[e * KW + kwo][g * 8 + (k & 7)][t];
      sum.x += v.x;
      sum.y += v.y;
    }
    part[((size_t)b * nblk + blockIdx.x) * KS + o] = sum;
  }
  finish_reduce(part, out, counter, KS, nblk, b);
}

// runs of QR consecutive complex values starting at an aligned address
template <int QR, typename C>
__device__ __forceinline__ void load_run(const C* p, C (&v)[QR]) {
  if constexpr (QR == 4) {
    load4(p, v);
  } else if constexpr (QR == 2 && sizeof(C) == 8) {
    const float4 a = reinterpret_cast<const float4*>(p)[0];  // two complex FP32 values, 16-byte aligned
    v[0] = make_float2(a.x, a.y);
    v[1] = make_float2(a.z, a.w);
  } else {
#pragma unroll
    for (int q = 0; q < QR; ++q) v[q] = p[q];
  }
}

// Z_t[b] = Y_t[b] - sum_k E[b][k*S + t] * X_k[b]  (FP64 tensor cores; S <= 16).  A warp owns 8*QR elements (lane
// gid: elements QR gid .. QR gid + QR - 1 of the tile) and runs over the basis 4 vectors at a time.  B tiles as in
// k_blockdot_mma; x c:  Re = P[t] - Q[4+t], Im = P[4+t] + Q[t]  (one tile) or, for t = 8h + c,
// Re = P[h][c] - Q[NTH + h][c],  Im = P[NTH + h][c] + Q[h][c].  Optional per-RHS basis sizes Kb[b] <= K.
//
// GRAM (S <= 8): the Gram matrix of the stored Z is accumulated on the way out, so that no second pass reads Z:
// out[b][tri(t,u)] = <Z_t, Z_u> for t <= u, tri(t,u) = t*S - t*(t-1)/2 + (u-t) (FP64, deterministic).  Each warp
// passes its tile through shared memory in two halves of 16 elements (lane (gid, tig) of the update holds elements
// 4 gid + q, columns 2 tig + i), and four k-steps of m8n8k4 MMAs per half take A = Z^H, B = Z with lane (gid, tig)
// holding Z[element tig of the k-step][column gid] for both operands.  Rows r of a half sit at r*8 + (t ^ gram_swz(r)),
// which keeps both the column-pair stores and the fragment loads free of bank conflicts.
__device__ __forceinline__ int gram_swz(int r) { return (2 * (r & 3)) ^ ((r >> 1) & 1); }

template <typename R, typename TY, int S, typename TZ = cplx<R>, bool GRAM = false>
__global__ void __launch_bounds__(KV_THREADS, 2) k_blockupdate_mma(long long M, int B, int K, const cplx<R>* U,
                                                                const TY* Y, TZ* Z,
                                                                const double2* __restrict__ coef,
                                                                const int* __restrict__ active,
                                                                const int* __restrict__ Kb = nullptr,
                                                                double2* __restrict__ gpart = nullptr,
                                                                double2* __restrict__ gout = nullptr,
                                                                unsigned* __restrict__ gcounter = nullptr) {
  static_assert(S >= 1 && S <= 16, "block update on tensor cores takes 1..16 block vectors");
  static_assert(!GRAM || S <= 8, "the fused Gram takes at most 8 block vectors");
  using T = cplx<R>;
  constexpr int NTH = S <= 4 ? 1 : (S + 7) / 8;
  constexpr int NT = S <= 4 ? 1 : 2 * NTH;
  constexpr int QR = S <= 8 ? 4 : 2;  // elements per lane (A rows of QR MMAs)
  constexpr int TILE = 8 * QR;        // elements per warp tile
  // coefficient rows padded to 4 (mod 16) doubles: the B-fragment loads (row kk + tig, column 8n + gid) then put
  // the four rows of a k-step 8 banks apart, two lanes per bank pair, the minimum for 256 bytes
  constexpr int BROW = (8 * NT + 15) / 16 * 16 + 4;
  __shared__ double Bs[KV_KMAX][BROW];
  __shared__ double2 zs[GRAM ? KV_WARPS * 128 : 1];       // one half tile (16 elements x 8 columns) per warp
  __shared__ double gacc[GRAM ? KV_WARPS * 4 * 32 : 1];  // per warp and lane: Re G[gid][2 tig + i], Im G[..]
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  if (Kb) K = Kb[b];
  if constexpr (GRAM) {
    for (int i = threadIdx.x; i < KV_WARPS * 4 * 32; i += blockDim.x) gacc[i] = 0.0;
  }
  for (int i = threadIdx.x; i < KV_KMAX * 8 * NT; i += blockDim.x) {
    const int k = i / (8 * NT), col = i - k * (8 * NT);
    int t;
    bool im;
    if constexpr (NT == 1) {
      t = col & 3;
      im = col >= 4;
    } else {
      im = col >= 8 * NTH;
      t = 8 * ((col >> 3) % NTH) + (col & 7);
    }
    double v = 0.0;
    if (k < K && t < S) {
      const double2 c = coef[(size_t)b * KV_KMAX * S + k * S + t];
      v = im ? c.y : c.x;
    }
    Bs[k][col] = v;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const size_t us = (size_t)B * M;
  const T* ub = U + (size_t)b * M;
  const TY* yb = Y + (size_t)b * M;
  TZ* zb = Z + (size_t)b * M;
  const long long tiles = (M + TILE - 1) / TILE;
  for (long long tl = (long long)blockIdx.x * KV_WARPS + w; tl < tiles; tl += (long long)gridDim.x * KV_WARPS) {
    const long long ea = tl * TILE + QR * gid;  // A rows of this lane: elements ea .. ea + QR - 1 (wholly in or out)
    const bool ein = ea < M;
    double P[QR][NT][2], Q[QR][NT][2];
#pragma unroll
    for (int q = 0; q < QR; ++q)
#pragma unroll
      for (int n = 0; n < NT; ++n) P[q][n][0] = P[q][n][1] = Q[q][n][0] = Q[q][n][1] = 0.0;
    // a ring of UPD_PD steps of basis loads (4 vectors each) stays in flight ahead of the MMAs
    constexpr int UPD_PD = 3;
    T xr[UPD_PD][QR];
#pragma unroll
    for (int r = 0; r < UPD_PD; ++r) {
#pragma unroll
      for (int q = 0; q < QR; ++q) {
        xr[r][q].x = 0;
        xr[r][q].y = 0;
      }
      const int kn = 4 * r + tig;
      if (kn < K && ein) load_run<QR>(ub + (size_t)kn * us + ea, xr[r]);
    }
    for (int k0 = 0; k0 < K; k0 += 4 * UPD_PD) {
#pragma unroll
      for (int r = 0; r < UPD_PD; ++r) {
        const int kk = k0 + 4 * r;
        if (kk >= K) break;  // warp-uniform
        T xv[QR];
#pragma unroll
        for (int q = 0; q < QR; ++q) {
          xv[q] = xr[r][q];
          xr[r][q].x = 0;
          xr[r][q].y = 0;
        }
        const int kn = kk + 4 * UPD_PD + tig;
        if (kn < K && ein) load_run<QR>(ub + (size_t)kn * us + ea, xr[r]);
        double bfr[NT];
#pragma unroll
        for (int n = 0; n < NT; ++n) bfr[n] = Bs[kk + tig][8 * n + gid];  // rows past K are zero
#pragma unroll
        for (int q = 0; q < QR; ++q) {
          const double2 x = to_d(xv[q]);
#pragma unroll
          for (int n = 0; n < NT; ++n) {
            mma_f64(P[q][n][0], P[q][n][1], x.x, bfr[n]);
            mma_f64(Q[q][n][0], Q[q][n][1], x.y, bfr[n]);
          }
        }
      }
    }
    // lane (gid, tig) holds C rows gid (element ea + q) and columns 2 tig, 2 tig + 1 of each tile
    double g[4] = {0.0, 0.0, 0.0, 0.0};  // this tile's Gram fragment (GRAM)
    double2* zw = zs + (GRAM ? w * 128 : 0);
#pragma unroll
    for (int q = 0; q < QR; ++q) {
      const long long e = ea + q;
      double2 zq[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};  // stored values of columns 2 tig + i
      if constexpr (NT == 1) {
        const double pp0 = __shfl_xor_sync(0xffffffffu, P[q][0][0], 2), pp1 = __shfl_xor_sync(0xffffffffu, P[q][0][1], 2);
        const double qp0 = __shfl_xor_sync(0xffffffffu, Q[q][0][0], 2), qp1 = __shfl_xor_sync(0xffffffffu, Q[q][0][1], 2);
        if (tig < 2 && ein) {
          const int t0 = 2 * tig;
          if (t0 < S) {
            const double2 y = to_d(yb[t0 * us + e]);
            const TZ z = from_d<TZ>(make_double2(y.x - (P[q][0][0] - qp0), y.y - (pp0 + Q[q][0][0])));
            zb[t0 * us + e] = z;
            zq[0] = to_d(z);
          }
          if (t0 + 1 < S) {
            const double2 y = to_d(yb[(t0 + 1) * us + e]);
            const TZ z = from_d<TZ>(make_double2(y.x - (P[q][0][1] - qp1), y.y - (pp1 + Q[q][0][1])));
            zb[(t0 + 1) * us + e] = z;
            zq[1] = to_d(z);
          }
        }
      } else if (ein) {
#pragma unroll
        for (int th = 0; th < NTH; ++th)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int t = 8 * th + 2 * tig + i;
            if (t < S) {
              const double2 y = to_d(yb[t * us + e]);
              const TZ z = from_d<TZ>(make_double2(y.x - (P[q][th][i] - Q[q][NTH + th][i]),
                                                   y.y - (P[q][NTH + th][i] + Q[q][th][i])));
              zb[t * us + e] = z;
              if (th == 0) zq[i] = to_d(z);
            }
          }
      }
      if constexpr (GRAM) {
        const int r = 2 * gid + (q & 1);  // row of element 4 gid + q in its half
#pragma unroll
        for (int i = 0; i < 2; ++i) zw[r * 8 + ((2 * tig + i) ^ gram_swz(r))] = zq[i];
        if (q & 1) {
          __syncwarp();
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int rr = 4 * j + tig;
            const double2 v = zw[rr * 8 + (gid ^ gram_swz(rr))];
            mma_f64(g[0], g[1], v.x, v.x);   // Re += zr_t zr_u
            mma_f64(g[0], g[1], v.y, v.y);   //    + zi_t zi_u
            mma_f64(g[2], g[3], v.x, v.y);   // Im += zr_t zi_u
            mma_f64(g[2], g[3], -v.y, v.x);  //    - zi_t zr_u
          }
          __syncwarp();
        }
      }
    }
    if constexpr (GRAM) {
      double* ga = gacc + w * 128 + lane;
#pragma unroll
      for (int c = 0; c < 4; ++c) ga[32 * c] += g[c];
    }
  }
  if constexpr (GRAM) {
    // CTA sum over the warps, then the grid-wide sum per RHS (deterministic order)
    constexpr int NG = S * (S + 1) / 2;
    __syncthreads();
    for (int o = threadIdx.x; o < NG; o += blockDim.x) {
      int t = 0, rem = o;
      while (rem >= S - t) {
        rem -= S - t;
        ++t;
      }
      const int u = t + rem, ln = 4 * t + (u >> 1), i = u & 1;
      double2 s = make_double2(0.0, 0.0);
      for (int q = 0; q < KV_WARPS; ++q) {
        s.x += gacc[q * 128 + 32 * i + ln];
        s.y += gacc[q * 128 + 32 * (2 + i) + ln];
      }
      gpart[((size_t)b * gridDim.x + blockIdx.x) * NG + o] = s;
    }
    finish_reduce(gpart, gout, gcounter, NG, gridDim.x, b);
  }
}

// Orthonormal block from the projected block vectors:  V_t[b] = sum_{u <= t} Z_u[b] c[b][u*S + t]
// (c = Rb^{-1}, upper triangular), Z in the block-vector type, V in the basis type.
template <typename R, typename TZ, int S>
__global__ void __launch_bounds__(KV_THREADS, 2) k_blocknorm(long long M, int B, const TZ* __restrict__ Z,
                                                          const double2* __restrict__ c, cplx<R>* __restrict__ V,
                                                          const int* __restrict__ active,
                                                          const int* __restrict__ vrow = nullptr) {
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  // coefficients are re-read from shared memory in the loop (volatile): held in registers they would take
  // S*S complex values per thread and halve the resident warps
  __shared__ double ccs[2 * S * S];
  volatile double* cc = ccs;
  if (threadIdx.x < S * S) {
    const double2 v = c[(size_t)b * S * S + threadIdx.x];
    ccs[2 * threadIdx.x] = v.x;
    ccs[2 * threadIdx.x + 1] = v.y;
  }
  __syncthreads();
  const size_t us = (size_t)B * M;
  const TZ* zb = Z + (size_t)b * M;
  cplx<R>* vb = V + (vrow ? (size_t)vrow[b] * us : 0) + (size_t)b * M;  // per-RHS first row (optional)
#pragma unroll 1
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < M; e += (long long)gridDim.x * blockDim.x) {
    double2 z[S];
#pragma unroll
    for (int u = 0; u < S; ++u) z[u] = to_d(zb[u * us + e]);
#pragma unroll
    for (int t = 0; t < S; ++t) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int u = 0; u <= t; ++u) {
        const double2 w = make_double2(cc[2 * (u * S + t)], cc[2 * (u * S + t) + 1]);
        acc.x = fma(w.x, z[u].x, fma(-w.y, z[u].y, acc.x));
        acc.y = fma(w.x, z[u].y, fma(w.y, z[u].x, acc.y));
      }
      vb[t * us + e] = from_d<cplx<R>>(acc);
    }
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
