// Register-resident, warp-synchronous Stockham FFT building blocks.
//
// A pencil of length L is held by TP = L/E consecutive lanes of one warp, E
// complex values per lane.  Each radix-R stage runs its butterflies in
// registers; between stages the pencil is exchanged through a small padded
// shared-memory buffer owned by the warp (no block-wide barrier).  The first
// stage reads its inputs straight from registers that the caller loaded from
// global memory, and the last stage leaves its outputs in registers in natural
// order, so global traffic is one read and one write per element.
//
// Register layout ("R-layout" for a stage of radix R):
//     v[m*R + q] = X[t + TP*m + q*(L/R)],   m in [0, E/R), q in [0, R)
// The forward FFT with radices (R0, R1, ...) consumes the R0-layout and yields
// the R_last-layout; the inverse is run with the radices reversed, so it
// consumes exactly what the forward produced and returns the R0-layout.
#pragma once
#include "fm_complex.cuh"

namespace fm {

// ---- radix butterflies (DIR = -1: exp(-i..) forward, +1: inverse, unnormalised) ----
template <int DIR, typename T>
__device__ __forceinline__ void bf2(T& a, T& b) {
  T t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int DIR, typename T>
__device__ __forceinline__ void bf4(T& v0, T& v1, T& v2, T& v3) {
  T t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = cmul_i<DIR>(csub(v1, v3));
  v0 = cadd(t0, t2);
  v2 = csub(t0, t2);
  v1 = cadd(t1, t3);
  v3 = csub(t1, t3);
}

// radix 3: X_k = sum_n v_n w^(nk), w = exp(DIR*2*pi*i/3) = -1/2 + i*DIR*sin(pi/3)
template <int DIR, typename T>
__device__ __forceinline__ void bf3(T& a, T& b, T& c) {
  using R = typename RealOf<T>::R;
  const R h = R(0.5), s3 = R(0.86602540378443864676);
  const T t1 = cadd(b, c), t2 = csub(b, c);
  const T m1 = mk(a.x - h * t1.x, a.y - h * t1.y);
  const T m2 = mk(-R(DIR) * s3 * t2.y, R(DIR) * s3 * t2.x);  // i*DIR*sin(pi/3)*(b - c)
  a = cadd(a, t1);
  b = cadd(m1, m2);
  c = csub(m1, m2);
}

// multiply by exp(DIR * 2*pi*i*M/16)
template <int DIR, int M, typename T>
__device__ __forceinline__ T tw16(T a) {
  using R = typename RealOf<T>::R;
  constexpr int m = M & 15;
  const R c1 = R(0.92387953251128675613), s1 = R(0.38268343236508977173), h = R(0.70710678118654752440);
  if constexpr (m == 0) return a;
  else if constexpr (m == 4) return cmul_i<DIR>(a);
  else if constexpr (m == 8) return mk(-a.x, -a.y);
  else if constexpr (m == 12) return cmul_i<-DIR>(a);
  else {
    R c, s;
    if constexpr (m == 1) { c = c1; s = s1; }
    else if constexpr (m == 2) { c = h; s = h; }
    else if constexpr (m == 3) { c = s1; s = c1; }
    else if constexpr (m == 5) { c = -s1; s = c1; }
    else if constexpr (m == 6) { c = -h; s = h; }
    else if constexpr (m == 7) { c = -c1; s = s1; }
    else if constexpr (m == 9) { c = -c1; s = -s1; }
    else if constexpr (m == 10) { c = -h; s = -h; }
    else if constexpr (m == 11) { c = -s1; s = -c1; }
    else if constexpr (m == 13) { c = s1; s = -c1; }
    else if constexpr (m == 14) { c = h; s = -h; }
    else { c = c1; s = -s1; }  // 15
    return cmul(a, mk(c, R(DIR) * s));
  }
}

template <int DIR, typename T>
__device__ __forceinline__ void bf8(T* v) {
  bf4<DIR>(v[0], v[2], v[4], v[6]);
  bf4<DIR>(v[1], v[3], v[5], v[7]);
  T o1 = tw16<DIR, 2>(v[3]), o2 = tw16<DIR, 4>(v[5]), o3 = tw16<DIR, 6>(v[7]);
  T e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int DIR, typename T>
__device__ __forceinline__ void bf16(T* v) {
  // n = 4*n1 + n2 ; k = k1 + 4*k2
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) bf4<DIR>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
  // v[n2 + 4*k1] *= w16^(n2*k1)
  v[5] = tw16<DIR, 1>(v[5]);  v[9] = tw16<DIR, 2>(v[9]);   v[13] = tw16<DIR, 3>(v[13]);
  v[6] = tw16<DIR, 2>(v[6]);  v[10] = tw16<DIR, 4>(v[10]); v[14] = tw16<DIR, 6>(v[14]);
  v[7] = tw16<DIR, 3>(v[7]);  v[11] = tw16<DIR, 6>(v[11]); v[15] = tw16<DIR, 9>(v[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) bf4<DIR>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // now v[4*k1 + k2] = X[k1 + 4*k2]; transpose to natural order
  T t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
}

template <int DIR, int RAD, typename T>
__device__ __forceinline__ void bfly(T* v) {
  if constexpr (RAD == 2) bf2<DIR>(v[0], v[1]);
  else if constexpr (RAD == 3) bf3<DIR>(v[0], v[1], v[2]);
  else if constexpr (RAD == 4) bf4<DIR>(v[0], v[1], v[2], v[3]);
  else if constexpr (RAD == 8) bf8<DIR>(v);
  else if constexpr (RAD == 16) bf16<DIR>(v);
  else static_assert(RAD == 2, "unsupported radix");
}

// ---- shared-memory exchange: one padding slot every 128 bytes of data ----
// (every 16 elements of float2, every 8 of double2), so the strided stage writes
// of consecutive lanes fall in distinct banks.
template <typename T>
__device__ __forceinline__ int sm_phys(int i) {
  return sizeof(T) == 16 ? i + (i >> 3) : i + (i >> 4);
}

// One Stockham stage: radix RAD, NS = product of the radices already applied.
// tw is the stage-twiddle table of the radix order being run: for the stage with
// prior product NS, entry (NS - 1) + (q - 1)*NS + k holds exp(-2*pi*i*k*q/(NS*RAD)),
// k in [0, NS), q in [1, RAD).  Consecutive lanes (consecutive k) read consecutive
// entries, and the stages together need exactly L - 1 entries.
template <int DIR, int L, int E, int RAD, int NS, bool LAST, typename T>
__device__ __forceinline__ void fft_stage(T (&v)[E], T* sm, const T* tw, int t) {
  constexpr int TP = L / E;
  constexpr int NB = E / RAD;
  static_assert(E % RAD == 0, "radix must divide E");
#pragma unroll
  for (int m = 0; m < NB; ++m) {
    const int j = t + TP * m;
    const int k = j % NS;
    if constexpr (NS > 1) {
#pragma unroll
      for (int q = 1; q < RAD; ++q) {
        T w = tw[(NS - 1) + (q - 1) * NS + k];
        if constexpr (DIR > 0) w = cconj(w);
        v[m * RAD + q] = cmul(v[m * RAD + q], w);
      }
    }
    bfly<DIR, RAD>(&v[m * RAD]);
    if constexpr (!LAST) {
      const int base = (j / NS) * NS * RAD + k;
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[sm_phys<T>(base + q * NS)] = v[m * RAD + q];
    }
  }
}

template <int L, int E, int RAD, typename T>
__device__ __forceinline__ void fft_gather(T (&v)[E], const T* sm, int t) {
  constexpr int TP = L / E;
#pragma unroll
  for (int m = 0; m < E / RAD; ++m)
#pragma unroll
    for (int q = 0; q < RAD; ++q) v[m * RAD + q] = sm[sm_phys<T>(t + TP * m + q * (L / RAD))];
}

// Full FFT of one pencil with the radix sequence (R0, R1, R2) (zeros = unused).
template <int DIR, int L, int E, int R0, int R1, int R2, typename T>
__device__ __forceinline__ void fft_run(T (&v)[E], T* sm, const T* tw, int t) {
  static_assert(R0 * (R1 ? R1 : 1) * (R2 ? R2 : 1) == L, "radices must multiply to L");
  if constexpr (R1 == 0) {
    fft_stage<DIR, L, E, R0, 1, true>(v, sm, tw, t);
  } else if constexpr (R2 == 0) {
    fft_stage<DIR, L, E, R0, 1, false>(v, sm, tw, t);
    __syncwarp();
    fft_gather<L, E, R1>(v, sm, t);
    __syncwarp();
    fft_stage<DIR, L, E, R1, R0, true>(v, sm, tw, t);
  } else {
    fft_stage<DIR, L, E, R0, 1, false>(v, sm, tw, t);
    __syncwarp();
    fft_gather<L, E, R1>(v, sm, t);
    __syncwarp();
    fft_stage<DIR, L, E, R1, R0, false>(v, sm, tw, t);
    __syncwarp();
    fft_gather<L, E, R2>(v, sm, t);
    __syncwarp();
    fft_stage<DIR, L, E, R2, R0 * R1, true>(v, sm, tw, t);
  }
}

// ---- NC pencils of one lane group run stage by stage together ----
// Pencil c exchanges through its own buffer sm + c*SMS, so between two __syncwarp the loads and butterflies of
// all NC pencils are independent and one pencil's exchange latency overlaps the others' arithmetic.  The stage
// twiddles are loaded once, before any store of the stage, and shared by the NC pencils.
template <int DIR, int L, int E, int RAD, int NS, bool LAST, int NC, int SMS, typename T>
__device__ __forceinline__ void fft_stage_n(T (&v)[NC][E], T* sm, const T* tw, int t) {
  constexpr int TP = L / E;
  constexpr int NB = E / RAD;
  static_assert(E % RAD == 0, "radix must divide E");
  T w[NB][RAD - 1];
  if constexpr (NS > 1) {
#pragma unroll
    for (int m = 0; m < NB; ++m)
#pragma unroll
      for (int q = 1; q < RAD; ++q) {
        T a = tw[(NS - 1) + (q - 1) * NS + (t + TP * m) % NS];
        if constexpr (DIR > 0) a = cconj(a);
        w[m][q - 1] = a;
      }
  }
#pragma unroll
  for (int m = 0; m < NB; ++m) {
    const int j = t + TP * m;
    const int k = j % NS;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if constexpr (NS > 1) {
#pragma unroll
        for (int q = 1; q < RAD; ++q) v[c][m * RAD + q] = cmul(v[c][m * RAD + q], w[m][q - 1]);
      }
      bfly<DIR, RAD>(&v[c][m * RAD]);
      if constexpr (!LAST) {
        const int base = (j / NS) * NS * RAD + k;
#pragma unroll
        for (int q = 0; q < RAD; ++q) sm[c * SMS + sm_phys<T>(base + q * NS)] = v[c][m * RAD + q];
      }
    }
  }
}

template <int L, int E, int RAD, int NC, int SMS, typename T>
__device__ __forceinline__ void fft_gather_n(T (&v)[NC][E], const T* sm, int t) {
#pragma unroll
  for (int c = 0; c < NC; ++c) fft_gather<L, E, RAD>(v[c], sm + c * SMS, t);
}

template <int DIR, int L, int E, int R0, int R1, int R2, int NC, int SMS, typename T>
__device__ __forceinline__ void fft_run_n(T (&v)[NC][E], T* sm, const T* tw, int t) {
  static_assert(R0 * (R1 ? R1 : 1) * (R2 ? R2 : 1) == L, "radices must multiply to L");
  if constexpr (R1 == 0) {
    fft_stage_n<DIR, L, E, R0, 1, true, NC, SMS>(v, sm, tw, t);
  } else if constexpr (R2 == 0) {
    fft_stage_n<DIR, L, E, R0, 1, false, NC, SMS>(v, sm, tw, t);
    __syncwarp();
    fft_gather_n<L, E, R1, NC, SMS>(v, sm, t);
    __syncwarp();
    fft_stage_n<DIR, L, E, R1, R0, true, NC, SMS>(v, sm, tw, t);
  } else {
    fft_stage_n<DIR, L, E, R0, 1, false, NC, SMS>(v, sm, tw, t);
    __syncwarp();
    fft_gather_n<L, E, R1, NC, SMS>(v, sm, t);
    __syncwarp();
    fft_stage_n<DIR, L, E, R1, R0, false, NC, SMS>(v, sm, tw, t);
    __syncwarp();
    fft_gather_n<L, E, R2, NC, SMS>(v, sm, t);
    __syncwarp();
    fft_stage_n<DIR, L, E, R2, R0 * R1, true, NC, SMS>(v, sm, tw, t);
  }
}

// ---- per-length plans ----
// E elements per lane and the forward radix sequence; TP = L/E lanes per pencil, 4 <= TP <= 32
// (so at most 8 pencils share a warp and every axis of >= 8 points tiles a warp).
template <int L, typename R> struct Plan;
#define FM_PLAN(LL, RT, EE, A, B, C)                                   \
  template <> struct Plan<LL, RT> {                                    \
    static constexpr int L = LL, E = EE, R0 = A, R1 = B, R2 = C;       \
    static constexpr int TP = LL / EE;                                 \
    static constexpr int RL = (C ? C : (B ? B : A)); /* last radix */  \
  };
FM_PLAN(8, float, 2, 2, 2, 2)
FM_PLAN(16, float, 4, 4, 4, 0)
FM_PLAN(32, float, 8, 8, 4, 0)
FM_PLAN(64, float, 8, 8, 8, 0)
FM_PLAN(128, float, 16, 16, 8, 0)
FM_PLAN(256, float, 16, 16, 16, 0)
FM_PLAN(512, float, 16, 16, 8, 4)
FM_PLAN(96, float, 24, 8, 4, 3)
FM_PLAN(8, double, 2, 2, 2, 2)
FM_PLAN(16, double, 4, 4, 4, 0)
FM_PLAN(32, double, 8, 8, 4, 0)
FM_PLAN(64, double, 8, 8, 8, 0)
FM_PLAN(128, double, 8, 8, 4, 4)
FM_PLAN(256, double, 8, 8, 8, 4)
FM_PLAN(512, double, 16, 16, 8, 4)
FM_PLAN(96, double, 24, 8, 4, 3)
#undef FM_PLAN

// forward-order run (radices R0, R1, R2) with its stage-twiddle table
template <int DIR, typename P, typename T>
__device__ __forceinline__ void fft_fwd_plan(T (&v)[P::E], T* sm, const T* tw_fwd, int t) {
  fft_run<DIR, P::L, P::E, P::R0, P::R1, P::R2>(v, sm, tw_fwd, t);
}
// reversed-order run (consumes the RL-layout, returns the R0-layout) with its own table
template <int DIR, typename P, typename T>
__device__ __forceinline__ void fft_rev_plan(T (&v)[P::E], T* sm, const T* tw_rev, int t) {
  if constexpr (P::R1 == 0) fft_run<DIR, P::L, P::E, P::R0, 0, 0>(v, sm, tw_rev, t);
  else if constexpr (P::R2 == 0) fft_run<DIR, P::L, P::E, P::R1, P::R0, 0>(v, sm, tw_rev, t);
  else fft_run<DIR, P::L, P::E, P::R2, P::R1, P::R0>(v, sm, tw_rev, t);
}

// NC pencils at once (exchange buffers SMS elements apart)
template <int DIR, typename P, int NC, int SMS, typename T>
__device__ __forceinline__ void fft_fwd_plan_n(T (&v)[NC][P::E], T* sm, const T* tw_fwd, int t) {
  fft_run_n<DIR, P::L, P::E, P::R0, P::R1, P::R2, NC, SMS>(v, sm, tw_fwd, t);
}
template <int DIR, typename P, int NC, int SMS, typename T>
__device__ __forceinline__ void fft_rev_plan_n(T (&v)[NC][P::E], T* sm, const T* tw_rev, int t) {
  if constexpr (P::R1 == 0) fft_run_n<DIR, P::L, P::E, P::R0, 0, 0, NC, SMS>(v, sm, tw_rev, t);
  else if constexpr (P::R2 == 0) fft_run_n<DIR, P::L, P::E, P::R1, P::R0, 0, NC, SMS>(v, sm, tw_rev, t);
  else fft_run_n<DIR, P::L, P::E, P::R2, P::R1, P::R0, NC, SMS>(v, sm, tw_rev, t);
}

// Padded pencil stride in the exchange buffer.  A shared-memory wavefront serves
// 128 bytes: 16 lanes of 8-byte or 8 lanes of 16-byte elements.  With lanes
// t-fastest (x rows) a wavefront spans 128/size/TP pencils, each using TP
// consecutive bank slots; with lanes pencil-fastest (y, z) it spans PW pencils
// with 128/size/PW slots each.  The stride is the padded length rounded up to
// the residue (mod 128 bytes) that puts those pencils on disjoint banks.
template <int L, typename T, int TP, bool TFAST>
struct PencilStride {
  static constexpr int units = 128 / (int)sizeof(T);
  static constexpr int base = sizeof(T) == 16 ? L + L / 8 : L + L / 16;
  static constexpr int PW = 32 / TP;
  static constexpr int r = TFAST ? (TP % units) : (PW >= units ? 0 : (units / PW) % units);
  static constexpr int v = base + ((r - base % units) % units + units) % units;
};

// index held in register e = m*R + q under the R-layout
template <int L, int E, int R>
__device__ __forceinline__ int lay_idx(int t, int e) {
  return t + (L / E) * (e / R) + (e % R) * (L / R);
}

}  // namespace fm
