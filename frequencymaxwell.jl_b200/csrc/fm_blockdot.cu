// Block dot D = X^H Y of block GMRES with a bulk-copy pipeline (FP64 tensor cores).
//
// Same result as k_blockdot_mma in fm_krylov.cuh (up to the order of the FP64 sums); the data path differs:
//
// * Work split.  The elements of all active right-hand sides form one list of 32-element units, cut into
//   gridDim.x equal contiguous ranges (one persistent CTA per SM).  A range touches at most two right-hand
//   sides, so every CTA does the same work whatever the batch size, and no SM idles when the number of
//   right-hand sides does not divide the SM count.
// * Pipeline.  A producer warp copies each chunk (C elements of the K basis vectors and of the S block
//   vectors) into a ring of NST shared-memory stages with cp.async.bulk (no cluster multicast), completing on
//   the stage's "full" mbarrier.  Eight consumer warps wait on it, read their fragments from shared memory,
//   run the m8n8k4 FP64 MMAs and arrive on the stage's "empty" mbarrier; the producer refills the stage after
//   that.  Global loads in flight no longer depend on how many registers the consumers hold.
// * Reduction.  When a CTA leaves a right-hand side its consumer warps sum their accumulators over the
//   sub-blocks of a chunk and write one partial per (CTA, slot).  The last contributing CTA (counter per
//   right-hand side) sums the partials of the contributing CTAs in CTA order, so the result does not depend
//   on timing.
//
// Every mbarrier wait is bounded.  A timed-out wait records a code in *err and sets a shared abort flag:
// from then on no warp waits, the producer issues nothing more, all warps still run the same sequence of
// named barriers, and the producer waits (bounded) for the copies it issued before the CTA exits.
#include "fm_blockdot.h"

#include <algorithm>
#include <type_traits>

#include "fm_krylov.cuh"
#include "fm_tma.cuh"

namespace fm {

namespace {

constexpr int BD_CW = 8;                      // consumer warps
constexpr int BD_THREADS = (BD_CW + 1) * 32;  // + one producer warp
constexpr int BD_GMAX = 4;                    // groups of 8 basis vectors per consumer warp, at most
// groups per consumer warp for S block vectors (two B tiles above S = 4 leave registers for two groups)
__host__ __device__ constexpr int bd_gmax(int S) { return S <= 4 ? 4 : 2; }
constexpr int BD_MAX_RHS = 2048;
constexpr int BD_SMEM_MAX = 227 * 1024;
constexpr int BD_MAX_STAGES = 6;

struct BdLayout {
  int C;           // elements per chunk (32 * 8 / WPS)
  int WPS;         // consumer warps per 32-element sub-block of a chunk
  int NST;         // stages
  int xrow, yrow;  // shared-memory bytes per basis / block row: C elements + 16 (conflict-free 128-bit reads)
  int stage;       // bytes per stage
  int red;         // offset of the reduction buffer
  int alist;       // offset of the list of active right-hand sides
  int bars;        // offset of the mbarriers (full[NST], empty[NST]) and three flag words
  int total;       // dynamic shared memory, including 128 bytes of alignment slack
};

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ long long ceil_div(long long a, long long b) { return (a + b - 1) / b; }

template <typename R, typename TY, int S>
__global__ void __launch_bounds__(BD_THREADS, 1)
    k_blockdot_bulk(long long M, int B, int K, const cplx<R>* __restrict__ U, const TY* __restrict__ Y,
                    double2* __restrict__ part, double2* __restrict__ out, unsigned* __restrict__ counter,
                    const int* __restrict__ active, int* __restrict__ err, BdLayout lay) {
  static_assert(S >= 1 && S <= 8, "block dot on tensor cores takes 1..8 block vectors");
  using T = cplx<R>;
  constexpr int NT = S <= 4 ? 1 : 2;  // 8-column B tiles, as in k_blockdot_mma
  constexpr int GM = bd_gmax(S);
  extern __shared__ unsigned char bd_raw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)bd_raw + 127) & ~(uintptr_t)127);
  int* alist = reinterpret_cast<int*>(sm + lay.alist);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + lay.bars);
  uint64_t* empty = full + lay.NST;
  volatile int* flags = reinterpret_cast<volatile int*>(empty + lay.NST);  // [0] active count, [1] abort, [2] last
  double2* red = reinterpret_cast<double2*>(sm + lay.red);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int NST = lay.NST;

  if (w == 0) {
    int cnt = 0;
    for (int b0 = 0; b0 < B; b0 += 32) {
      const int b = b0 + lane;
      const bool on = b < B && (!active || active[b]);
      const unsigned m = __ballot_sync(0xffffffffu, on);
      if (on) alist[cnt + __popc(m & ((1u << lane) - 1u))] = b;
      cnt += __popc(m);
    }
    if (lane == 0) {
      flags[0] = cnt;
      flags[1] = 0;
      for (int s = 0; s < NST; ++s) {
        mbar_init(full + s, 1);
        mbar_init(empty + s, BD_CW);
      }
      fence_barrier_init();
    }
  }
  __syncthreads();
  const long long nA = flags[0];
  const long long nun = (M + 31) / 32;  // 32-element units per right-hand side
  const long long UT = nA * nun;
  const long long G = gridDim.x;
  if (nA == 0) return;
  if (G > UT || G < nA) {  // the launcher sizes the grid inside [nA, UT]
    if (tid == 0) atomicExch(err, 31);
    return;
  }
  const long long u0 = (long long)blockIdx.x * UT / G, u1 = ((long long)blockIdx.x + 1) * UT / G;
  const int CU = lay.C / 32;
  const size_t us = (size_t)B * M;
  const int KS = K * S;

  // chunk at unit u of this CTA's range: right-hand side (compact index) j, first element e0, n elements
  auto chunk = [&](long long u, long long& j, long long& e0, int& n, int& cu) {
    j = u / nun;
    const long long seg = min(u1, (j + 1) * nun);
    cu = (int)min((long long)CU, seg - u);
    e0 = (u - j * nun) * 32;
    n = (int)min((long long)cu * 32, M - e0);
  };

  if (w == BD_CW) {
    // ------------------------------------------------------------------ producer warp
    int it = 0;
    for (long long u = u0; u < u1; ++it) {
      long long j, e0;
      int n, cu;
      chunk(u, j, e0, n, cu);
      const int s = it % NST;
      int stop = 0;
      if (lane == 0) {  // lane 0 decides for the warp: no divergent exit
        if (it >= NST && !flags[1] && !mbar_wait(empty + s, ((it / NST) - 1) & 1, err, 32)) flags[1] = 1;
        stop = flags[1];
      }
      if (__shfl_sync(0xffffffffu, stop, 0)) break;
      const int b = alist[j];
      unsigned char* st = sm + (size_t)s * lay.stage;
      if (lane == 0) mbar_expect_tx(full + s, (uint32_t)n * (uint32_t)(K * sizeof(T) + S * sizeof(TY)));
      __syncwarp();
      for (int r = lane; r < K + S; r += 32) {
        if (r < K)
          bulk_g2s(st + (size_t)r * lay.xrow, U + (size_t)r * us + (size_t)b * M + e0, (uint32_t)(n * sizeof(T)),
                   full + s);
        else
          bulk_g2s(st + (size_t)K * lay.xrow + (size_t)(r - K) * lay.yrow,
                   Y + (size_t)(r - K) * us + (size_t)b * M + e0, (uint32_t)(n * sizeof(TY)), full + s);
      }
      u += cu;
    }
    // wait (bounded) until every copy this warp issued has landed
    if (lane == 0)
      for (int k = 0; k < NST && k < it; ++k) {
        const int i = it - 1 - k;
        mbar_wait(full + (i % NST), (i / NST) & 1, err, 33);
      }
    return;
  }

  // -------------------------------------------------------------------- consumer warps
  const int gid = lane >> 2, tig = lane & 3;
  const int WPS = lay.WPS, NSUB = BD_CW / WPS;
  const int sub = w / WPS, rw = w % WPS;
  const int KG = (K + 7) >> 3;
  const int yt = NT == 1 ? (gid & 3) : gid;  // block vector of this lane's B column
  const bool yon = yt < S;
  double P[BD_GMAX][NT][2], Q[BD_GMAX][NT][2];
  auto zero = [&]() {
#pragma unroll
    for (int g = 0; g < BD_GMAX; ++g)
#pragma unroll
      for (int t = 0; t < NT; ++t) P[g][t][0] = P[g][t][1] = Q[g][t][0] = Q[g][t][1] = 0.0;
  };
  zero();

  // sum this CTA's accumulators for right-hand side (compact index) j into its partial; the last contributor
  // reduces the partials of all contributors, in CTA order, into out
  auto flush = [&](long long j) {
#pragma unroll
    for (int jg = 0; jg < GM; ++jg) {
      const int g = rw + jg * WPS;
      if (g >= KG) break;
      double2* rr = red + ((size_t)(w * BD_GMAX + jg) * 8 + gid) * S;
      if constexpr (NT == 1) {
        // columns 2 tig, 2 tig + 1 hold Re Y; the partner lane tig ^ 2 holds the Im Y columns 4 + ...
        const double pp0 = __shfl_xor_sync(0xffffffffu, P[jg][0][0], 2);
        const double pp1 = __shfl_xor_sync(0xffffffffu, P[jg][0][1], 2);
        const double qp0 = __shfl_xor_sync(0xffffffffu, Q[jg][0][0], 2);
        const double qp1 = __shfl_xor_sync(0xffffffffu, Q[jg][0][1], 2);
        if (tig < 2) {
          const int t0 = 2 * tig;
          if (t0 < S) rr[t0] = make_double2(P[jg][0][0] + qp0, pp0 - Q[jg][0][0]);
          if (t0 + 1 < S) rr[t0 + 1] = make_double2(P[jg][0][1] + qp1, pp1 - Q[jg][0][1]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int t = 2 * tig + i;
          if (t < S) rr[t] = make_double2(P[jg][0][i] + Q[jg][NT - 1][i], P[jg][NT - 1][i] - Q[jg][0][i]);
        }
      }
    }
    named_bar(1, BD_CW * 32);
    const int slot = (int)(j - u0 / nun);
    double2* mine = part + ((size_t)blockIdx.x * 2 + slot) * KS;
    for (int o = tid; o < KS; o += BD_CW * 32) {
      const int k = o / S, t = o - k * S;
      const int g = k >> 3, r = g % WPS, jg = g / WPS;
      double2 sum = make_double2(0.0, 0.0);
      for (int sb = 0; sb < NSUB; ++sb) {
        const double2 v = red[((size_t)((sb * WPS + r) * BD_GMAX + jg) * 8 + (k & 7)) * S + t];
        sum.x += v.x;
        sum.y += v.y;
      }
      mine[o] = sum;
    }
    __threadfence();
    named_bar(1, BD_CW * 32);
    const long long c_lo = ceil_div((j * nun + 1) * G, UT) - 1;
    const long long c_hi = ceil_div((j + 1) * nun * G, UT) - 1;
    const int b = alist[j];
    if (tid == 0) {
      const unsigned tk = atomicAdd(&counter[b], 1u);
      flags[2] = (tk == (unsigned)(c_hi - c_lo));
    }
    named_bar(1, BD_CW * 32);
    if (flags[2]) {
      __threadfence();
      for (int o = tid; o < KS; o += BD_CW * 32) {
        double2 sum = make_double2(0.0, 0.0);
        for (long long c = c_lo; c <= c_hi; ++c) {
          const int sc = (int)(j - (c * UT / G) / nun);
          const double2 v = __ldcg(&part[((size_t)c * 2 + sc) * KS + o]);
          sum.x += v.x;
          sum.y += v.y;
        }
        out[(size_t)b * KS + o] = sum;
      }
      if (tid == 0) counter[b] = 0;
    }
    named_bar(1, BD_CW * 32);
    zero();
  };

  int it = 0;
  long long jcur = -1;
  for (long long u = u0; u < u1; ++it) {
    long long j, e0;
    int n, cu;
    chunk(u, j, e0, n, cu);
    if (j != jcur) {
      if (jcur >= 0) flush(jcur);
      jcur = j;
    }
    const int s = it % NST;
    if (lane == 0 && !flags[1] && !mbar_wait(full + s, (it / NST) & 1, err, 34)) flags[1] = 1;
    __syncwarp();
    const unsigned char* st = sm + (size_t)s * lay.stage;
    const int eb = sub * 32;
    if (eb < n) {
      const TY* yrow = reinterpret_cast<const TY*>(st + (size_t)K * lay.xrow + (size_t)(yon ? yt : 0) * lay.yrow);
      double bf[NT][2][4];
      bool ein[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int el = eb + 16 * h + 4 * tig;  // runs of 4 lie wholly inside or outside the chunk
        ein[h] = el < n;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          double2 y = make_double2(0.0, 0.0);
          if (yon && ein[h]) y = to_d(yrow[el + q]);
          if constexpr (NT == 1) {
            bf[0][h][q] = gid >= 4 ? y.y : y.x;
          } else {
            bf[0][h][q] = y.x;
            bf[NT - 1][h][q] = y.y;
          }
        }
      }
      // all groups' fragments first, then the MMAs with the groups innermost: 2 NG independent accumulator
      // chains per warp keep the FP64 tensor pipe busy (one group at a time leaves it waiting on MMA latency)
      auto tile = [&](auto ngc) {
        constexpr int NG = decltype(ngc)::value;
        T xv[NG][2][4];
#pragma unroll
        for (int jg = 0; jg < NG; ++jg) {
          const int k = (rw + jg * WPS) * 8 + gid;
          const T* xrow = reinterpret_cast<const T*>(st + (size_t)(k < K ? k : 0) * lay.xrow);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              xv[jg][h][q].x = 0;
              xv[jg][h][q].y = 0;
            }
            if (k < K && ein[h]) load4(xrow + eb + 16 * h + 4 * tig, xv[jg][h]);
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int jg = 0; jg < NG; ++jg) {
              const double2 x = to_d(xv[jg][h][q]);
#pragma unroll
              for (int t = 0; t < NT; ++t) {
                mma_f64(P[jg][t][0], P[jg][t][1], x.x, bf[t][h][q]);
                mma_f64(Q[jg][t][0], Q[jg][t][1], x.y, bf[t][h][q]);
              }
            }
      };
      const int ng = KG > rw ? min(GM, (KG - rw + WPS - 1) / WPS) : 0;  // warp-uniform
      switch (ng) {
        case 1: tile(std::integral_constant<int, 1>{}); break;
        case 2: tile(std::integral_constant<int, 2>{}); break;
        case 3: if constexpr (GM >= 3) tile(std::integral_constant<int, 3>{}); break;
        case 4: if constexpr (GM >= 4) tile(std::integral_constant<int, 4>{}); break;
        default: break;
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(empty + s);
    u += cu;
  }
  if (jcur >= 0) flush(jcur);
}

bool bd_layout(int K, int S, int tb, int yb, int nb, BdLayout& L) {
  if (K < 1 || K > KV_KMAX || S < 1 || S > 8 || nb < 1 || nb > BD_MAX_RHS) return false;
  const int KG = (K + 7) / 8;
  int wps = 1;
  const int gm = bd_gmax(S);
  while (wps < BD_CW && (KG + wps - 1) / wps > gm) wps *= 2;
  if ((KG + wps - 1) / wps > gm) return false;
  const int redb = BD_CW * BD_GMAX * 8 * S * (int)sizeof(double2);
  const int alb = ((nb * 4 + 15) / 16) * 16;
  const int fixed = 128 + redb + alb + 2 * BD_MAX_STAGES * 8 + 16;
  // largest chunk that still leaves three stages (two at the smallest chunk)
  for (;; wps *= 2) {
    L.WPS = wps;
    L.C = 32 * (BD_CW / wps);
    L.xrow = L.C * tb + 16;
    L.yrow = L.C * yb + 16;
    L.stage = ((K * L.xrow + S * L.yrow) + 127) / 128 * 128;
    L.NST = std::min(BD_MAX_STAGES, (BD_SMEM_MAX - fixed) / L.stage);
    if (L.NST >= 3 || wps == BD_CW) break;
  }
  if (L.NST < 2) return false;
  L.red = L.NST * L.stage;
  L.alist = L.red + redb;
  L.bars = L.alist + alb;
  L.total = 128 + L.bars + 2 * L.NST * 8 + 16;
  return L.total <= BD_SMEM_MAX;
}

long long bd_grid(long long M, int nact, int sms) {
  const long long UT = (long long)nact * ((M + 31) / 32);
  return std::min(std::max<long long>(sms, nact), UT);
}

template <typename R, typename TY, int S>
cudaError_t launch_S(long long M, int nb, int nact, int K, const void* U, const void* Y, double2* part, size_t pbytes,
                     double2* out, unsigned* counter, const int* act, int* err, int sms, cudaStream_t st) {
  BdLayout L;
  if (!bd_layout(K, S, (int)sizeof(cplx<R>), (int)sizeof(TY), nb, L)) return cudaErrorNotSupported;
  if (nact < 1) return cudaSuccess;
  const long long G = bd_grid(M, nact, sms);
  if ((size_t)G * 2 * K * S * sizeof(double2) > pbytes) return cudaErrorInvalidValue;
  auto kern = k_blockdot_bulk<R, TY, S>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)G, BD_THREADS, L.total, st>>>(M, nb, K, (const cplx<R>*)U, (const TY*)Y, part, out, counter, act,
                                                 err, L);
  return cudaGetLastError();
}

template <typename R, typename TY>
cudaError_t launch_T(int S, long long M, int nb, int nact, int K, const void* U, const void* Y, double2* part,
                     size_t pbytes, double2* out, unsigned* counter, const int* act, int* err, int sms,
                     cudaStream_t st) {
  switch (S) {
#define BD_CASE(s) \
  case s: return launch_S<R, TY, s>(M, nb, nact, K, U, Y, part, pbytes, out, counter, act, err, sms, st);
    BD_CASE(2) BD_CASE(3) BD_CASE(4) BD_CASE(5) BD_CASE(6) BD_CASE(7) BD_CASE(8)
#undef BD_CASE
    default: return cudaErrorNotSupported;
  }
}

bool types_ok(int rbytes, int ybytes) {
  return (rbytes == 4 && (ybytes == 4 || ybytes == 8)) || (rbytes == 8 && ybytes == 8);
}

}  // namespace

size_t blockdot_bulk_part_bytes(int rbytes, int ybytes, int S, long long M, int nb, int nact, int K, int sms) {
  BdLayout L;
  if (!types_ok(rbytes, ybytes) || (M & 3) != 0 || S < 2 || S > 8 || !bd_layout(K, S, 2 * rbytes, 2 * ybytes, nb, L))
    return 0;
  return (size_t)std::max<long long>(1, bd_grid(M, std::max(nact, 1), sms)) * 2 * K * S * sizeof(double2);
}

cudaError_t launch_blockdot_bulk(int rbytes, int ybytes, int S, long long M, int nb, int nact, int K, const void* U,
                                 const void* Y, double2* part, size_t pbytes, double2* out, unsigned* counter,
                                 const int* act, int* err, int sms, cudaStream_t st) {
  if ((M & 3) != 0 || !types_ok(rbytes, ybytes)) return cudaErrorNotSupported;
  if (rbytes == 4 && ybytes == 8)
    return launch_T<float, double2>(S, M, nb, nact, K, U, Y, part, pbytes, out, counter, act, err, sms, st);
  if (rbytes == 4)
    return launch_T<float, float2>(S, M, nb, nact, K, U, Y, part, pbytes, out, counter, act, err, sms, st);
  return launch_T<double, double2>(S, M, nb, nact, K, U, Y, part, pbytes, out, counter, act, err, sms, st);
}

}  // namespace fm
