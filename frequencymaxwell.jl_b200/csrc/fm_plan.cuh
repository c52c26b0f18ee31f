// libfmcuda internals shared by its translation units: the plan object, workspace buffers, kernel accounting,
// pass dispatch, tables, and the declarations of the operator drivers (fm_ops.cu), the Krylov drivers
// (fm_gmres.cu), the slot engine (fm_engine.cu) and the C ABI (fm_capi.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <memory>
#include <deque>
#include <future>
#include <thread>
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fmcuda.h"
#include "fm_blockdot.h"
#include "fm_krylov.cuh"
#include "fm_generic.h"
#include "fm_launch.h"
#include "fm_setup.cuh"
#include "fm_tables.h"

using namespace fm;
using cd = std::complex<double>;

extern thread_local std::string g_err;  // message of the last failure on this thread (fm_capi.cu)


inline fm_status fail(fm_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

#define FM_CK(expr)                                                                              \
  do {                                                                                           \
    cudaError_t e_ = (expr);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      return fail(e_ == cudaErrorMemoryAllocation ? FM_ERR_OOM : FM_ERR_CUDA,                    \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                          \
    }                                                                                            \
  } while (0)

#define FM_TRY(expr)               \
  do {                             \
    fm_status s_ = (expr);         \
    if (s_ != FM_OK) return s_;    \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct fm_plan {
  fm_plan_desc desc{};
  int prec = FM_PREC_F32;
  size_t esz = 8;  // bytes per complex element in HBM
  bool c64 = false;  // FFT / Green / V arithmetic in FP64 (FP64 storage, or FP32 storage with FP64 math)
  Dims dims{};
  PadInfo pi{};
  long long n = 0, M = 0;  // voxels, elements per field (3n)
  cudaStream_t st = nullptr;
  int sms = 148;
  bool use_tma = true;  // TMA-staged y/z passes (FMCUDA_NO_TMA=1 selects the register-only passes)
  bool tma_y = true, tma_z = true;  // tuning: TMA-staged y / z passes where the size has one
  bool bd_bulk = false;             // tuning: bulk-copy pipelined block dot where the shape has one
  bool bd_wide = false;             // tuning: register block dot with four basis groups per warp (5 <= s <= 8)
  int wave_rhs = 0;                 // tuning: right-hand sides per wave at most (0: as many as memory holds)
  DevBuf errbuf;        // device error code written by bounded pipeline waits
  bool avg = false;     // any absorbing axis
  bool zonly = false;   // shifts only on z -> single pass with the length-2L transform
  bool zsplit = false;  // shifts only on z, padded z longer than the length-2L pass takes: two z passes
  bool generic = false; // an axis without a fused pass (fm_generic.cuh): plain passes, Bluestein where needed
  GenAxis gax[3];       // device tables of the general passes per axis
  DevBuf gtw[3], gch[3][2], gkn[3][2];
  double shift[3] = {0, 0, 0};
  // potential / physics
  bool have_pot = false;
  double k_bg = 0, eps_imag = 0, wavelength = 0, kref2 = 1;
  int bornmax = 0;
  // tables (plan precision)
  DevBuf twx, twy, twz, twz2, rz, rxp, rxm, ryp, rym, rzp, rzm;
  DevBuf V;
  // workspace
  DevBuf t1, t2, t3, bbuf, xbuf, ebuf, sbuf, basis, gbuf2;  // t3: first branch of a two-branch average
  DevBuf red_part, red_out, red_cnt, active, scale, coef, hbuf, shifts, yblk, V64;
  DevBuf eps_dev, fx, fy, fz, maxpart, maxout;
  bool eps_phantom = false;  // eps_dev holds the permittivity fm_phantom_fill painted (fm_build_potential eps = NULL)
  DevBuf shapes;             // fm_phantom_fill's shape table
  DevBuf wt_x, wt_y, wt_z, wt_pe, wt_ph, wt_first;
  DevBuf Eo, Ho;
  int out_nrhs = 0;
  // copies of the output fields to the caller's host buffers (solve_waves_t): a copy stream, a pinned staging
  // ring of two chunks, "chunk landed" events and "output slot assembled" events
  cudaStream_t cst = nullptr;
  void* stage_h = nullptr;
  cudaEvent_t cev[2] = {nullptr, nullptr};
  cudaEvent_t ready[2] = {nullptr, nullptr};
  // launch accounting (always) and event timing per kernel class (when prof is on)
  bool prof = false;
  long long launches[16] = {0};
  double kms[16] = {0}, kbytes[16] = {0};
  long long total_launches = 0;
  struct Pending { int cls; double bytes; cudaEvent_t a, b; };
  std::vector<Pending> pend;
  std::vector<cudaEvent_t> evpool;
};

// ---------------------------------------------------------------------------
// kernel accounting
// ---------------------------------------------------------------------------
enum KCls { KC_XF = 0, KC_YF, KC_ZG, KC_YI, KC_XI, KC_DOT, KC_UPD, KC_MGS, KC_AXPBY, KC_CURL, KC_SETUP, KC_N };
static const char* const kcls_name[KC_N] = {"xf", "yf", "zg", "yi", "xi", "multidot", "update", "mgs/gram", "axpby", "curl", "setup"};

inline cudaEvent_t ev_get(fm_plan* P) {
  if (!P->evpool.empty()) {
    cudaEvent_t e = P->evpool.back();
    P->evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

inline void tk_resolve(fm_plan* P) {
  for (auto& q : P->pend) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, q.a, q.b) == cudaSuccess) {
      P->kms[q.cls] += ms;
      P->kbytes[q.cls] += q.bytes;
    }
    P->evpool.push_back(q.a);
    P->evpool.push_back(q.b);
  }
  P->pend.clear();
}

struct Tk {
  fm_plan* P;
  int cls;
  double bytes;
  cudaEvent_t a;
};
inline Tk tk_begin(fm_plan* P, int cls, double bytes) {
  Tk t{P, cls, bytes, nullptr};
  if (P->prof) {
    if (P->pend.size() > 8192) {  // bound the number of outstanding events
      cudaStreamSynchronize(P->st);
      tk_resolve(P);
    }
    t.a = ev_get(P);
    cudaEventRecord(t.a, P->st);
  }
  return t;
}
inline void tk_end(const Tk& t) {
  t.P->launches[t.cls]++;
  t.P->total_launches++;
  if (t.P->prof) {
    cudaEvent_t b = ev_get(t.P);
    cudaEventRecord(b, t.P->st);
    t.P->pend.push_back({t.cls, t.bytes, t.a, b});
  }
}
#define FM_TRACK(P, cls, bytes, stmt)          \
  do {                                         \
    Tk tk_ = tk_begin((P), (cls), (bytes));    \
    stmt;                                      \
    tk_end(tk_);                               \
  } while (0)

// ---------------------------------------------------------------------------
// pass dispatch: storage type S, arithmetic double when the plan asks for it
// ---------------------------------------------------------------------------
template <typename S>
static cudaError_t pass_xf(const fm_plan* P, const Dims& d, int pro, const void* in, const void* V, const double* rs,
                           const void* tw, const void* ramp, void* out, const int* act, VecTab vt = VecTab{}) {
  if constexpr (std::is_same<S, double>::value)
    return launch_xf<double, double>(d, pro, in, V, rs, tw, ramp, out, act, P->st, vt);
  else return P->c64 ? launch_xf<float, double>(d, pro, in, V, rs, tw, ramp, out, act, P->st, vt)
                     : launch_xf<float, float>(d, pro, in, V, rs, tw, ramp, out, act, P->st, vt);
}
template <typename S>
static cudaError_t pass_y(const fm_plan* P, const Dims& d, int dir, const void* in, const void* tw, const void* ramp,
                          void* out, const int* act) {
  if (P->use_tma && P->tma_y && !ramp) {
    cudaError_t e;
    if constexpr (std::is_same<S, double>::value)
      e = launch_y_tma<double, double>(d, dir, in, tw, ramp, out, act, (int*)P->errbuf.p, P->sms, P->st);
    else
      e = P->c64 ? launch_y_tma<float, double>(d, dir, in, tw, ramp, out, act, (int*)P->errbuf.p, P->sms, P->st)
                 : launch_y_tma<float, float>(d, dir, in, tw, ramp, out, act, (int*)P->errbuf.p, P->sms, P->st);
    if (e != cudaErrorNotSupported) return e;
  }
  if constexpr (std::is_same<S, double>::value) return launch_y<double, double>(d, dir, in, tw, ramp, out, act, P->st);
  else return P->c64 ? launch_y<float, double>(d, dir, in, tw, ramp, out, act, P->st)
                     : launch_y<float, float>(d, dir, in, tw, ramp, out, act, P->st);
}
template <typename S>
static cudaError_t pass_zg(const fm_plan* P, const Dims& d, int mode, const void* in, const GreenParams& gp,
                           const void* tw, const void* rz, void* out, const int* act) {
  if (P->use_tma && P->tma_z) {
    cudaError_t e;
    if constexpr (std::is_same<S, double>::value)
      e = launch_zg_tma<double, double>(d, mode, in, gp, tw, rz, out, act, (int*)P->errbuf.p, P->sms, P->st);
    else
      e = P->c64 ? launch_zg_tma<float, double>(d, mode, in, gp, tw, rz, out, act, (int*)P->errbuf.p, P->sms, P->st)
                 : launch_zg_tma<float, float>(d, mode, in, gp, tw, rz, out, act, (int*)P->errbuf.p, P->sms, P->st);
    if (e != cudaErrorNotSupported) return e;
  }
  if constexpr (std::is_same<S, double>::value) return launch_zg<double, double>(d, mode, in, gp, tw, rz, out, act, P->st);
  else return P->c64 ? launch_zg<float, double>(d, mode, in, gp, tw, rz, out, act, P->st)
                     : launch_zg<float, float>(d, mode, in, gp, tw, rz, out, act, P->st);
}
template <typename S>
static cudaError_t pass_xi(const fm_plan* P, const Dims& d, int epi, const void* in, const void* V, const void* xv,
                           const void* bv, const double* rs, const EpiParams& ep, const void* tw, const void* ramp,
                           void* out, const int* act, VecTab vt = VecTab{}) {
  if constexpr (std::is_same<S, double>::value)
    return launch_xi<double, double>(d, epi, in, V, xv, bv, rs, ep, tw, ramp, out, act, P->st, vt);
  else return P->c64 ? launch_xi<float, double>(d, epi, in, V, xv, bv, rs, ep, tw, ramp, out, act, P->st, vt)
                     : launch_xi<float, float>(d, epi, in, V, xv, bv, rs, ep, tw, ramp, out, act, P->st, vt);
}
template <typename S>
static cudaError_t pass_xi_xf(const fm_plan* P, const Dims& d, const void* in, const void* V, const void* xv,
                              const EpiParams& ep, const void* tw, void* out, void* out2, const int* act) {
  if constexpr (std::is_same<S, double>::value)
    return launch_xi_xf<double, double>(d, in, V, xv, ep, tw, out, out2, act, P->st);
  else return P->c64 ? launch_xi_xf<float, double>(d, in, V, xv, ep, tw, out, out2, act, P->st)
                     : launch_xi_xf<float, float>(d, in, V, xv, ep, tw, out, out2, act, P->st);
}

// ---------------------------------------------------------------------------
// tables
// ---------------------------------------------------------------------------
template <typename R>
static cudaError_t upload_cplx(DevBuf& buf, const std::vector<cd>& v, cudaStream_t st) {
  using T = cplx<R>;
  std::vector<T> h(v.size());
  for (size_t i = 0; i < v.size(); ++i) h[i] = mk((R)v[i].real(), (R)v[i].imag());
  cudaError_t e = buf.ensure(std::max<size_t>(1, h.size()) * sizeof(T));
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(buf.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

template <typename R>
static fm_status init_tables(fm_plan* P) {
  if (P->generic) {
    const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
    for (int a = 0; a < 3; ++a) {
      const GenAxisTables t = gen_axis_tables(n3[a]);
      GenAxis& g = P->gax[a];
      g.n = t.n;
      g.m = t.m;
      FM_CK(upload_cplx<R>(P->gtw[a], twiddles<R>(t.m), P->st));
      g.tw = P->gtw[a].p;
      if (t.m != t.n) {
        for (int dir = 0; dir < 2; ++dir) {
          FM_CK(upload_cplx<R>(P->gch[a][dir], t.chirp[dir], P->st));
          FM_CK(upload_cplx<R>(P->gkn[a][dir], t.kern[dir], P->st));
          g.chirp[dir] = P->gch[a][dir].p;
          g.kern[dir] = P->gkn[a][dir].p;
        }
      }
    }
    if (P->avg) {
      FM_CK(upload_cplx<R>(P->rxp, ramp(P->dims.nx, P->shift[0], -1.0), P->st));
      FM_CK(upload_cplx<R>(P->rxm, ramp(P->dims.nx, P->shift[0], +1.0), P->st));
      FM_CK(upload_cplx<R>(P->ryp, ramp(P->dims.ny, P->shift[1], -1.0), P->st));
      FM_CK(upload_cplx<R>(P->rym, ramp(P->dims.ny, P->shift[1], +1.0), P->st));
      FM_CK(upload_cplx<R>(P->rzp, ramp(P->dims.nz, P->shift[2], -1.0), P->st));
      FM_CK(upload_cplx<R>(P->rzm, ramp(P->dims.nz, P->shift[2], +1.0), P->st));
    }
    return FM_OK;
  }
  FM_CK(upload_cplx<R>(P->twx, twiddles<R>(P->dims.nx), P->st));
  FM_CK(upload_cplx<R>(P->twy, twiddles<R>(P->dims.ny), P->st));
  FM_CK(upload_cplx<R>(P->twz, twiddles<R>(P->dims.nz), P->st));
  if (P->zonly) {
    FM_CK(upload_cplx<R>(P->twz2, twiddles<R>(2 * P->dims.nz), P->st));
    FM_CK(upload_cplx<R>(P->rz, ramp(P->dims.nz, P->shift[2], -1.0), P->st));
  } else if (P->zsplit) {
    FM_CK(upload_cplx<R>(P->rzp, ramp(P->dims.nz, P->shift[2], -1.0), P->st));
    FM_CK(upload_cplx<R>(P->rzm, ramp(P->dims.nz, P->shift[2], +1.0), P->st));
  } else if (P->avg) {
    FM_CK(upload_cplx<R>(P->rxp, ramp(P->dims.nx, P->shift[0], -1.0), P->st));
    FM_CK(upload_cplx<R>(P->rxm, ramp(P->dims.nx, P->shift[0], +1.0), P->st));
    FM_CK(upload_cplx<R>(P->ryp, ramp(P->dims.ny, P->shift[1], -1.0), P->st));
    FM_CK(upload_cplx<R>(P->rym, ramp(P->dims.ny, P->shift[1], +1.0), P->st));
    FM_CK(upload_cplx<R>(P->rzp, ramp(P->dims.nz, P->shift[2], -1.0), P->st));
    FM_CK(upload_cplx<R>(P->rzm, ramp(P->dims.nz, P->shift[2], +1.0), P->st));
  }
  return FM_OK;
}

// ---------------------------------------------------------------------------
// workspace
// ---------------------------------------------------------------------------
// Blocks per RHS for a Krylov kernel: one full wave of resident blocks
// (SMs x occupancy) shared by the nb right-hand sides, so no launch ends with a
// partly filled second wave.
template <typename Kern>
static int kv_blocks(const fm_plan* P, Kern kern, int nb) {
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, KV_THREADS, 0) != cudaSuccess || bps < 1) bps = 1;
  const long long cap = (long long)P->sms * bps;
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long maxb = (P->M + chunk - 1) / chunk;
  return (int)std::max(1LL, std::min<long long>(maxb, cap / nb));
}
inline int red_blocks_max(const fm_plan* P, int nb) {
  // upper bound of kv_blocks over all kernels (at most 8 blocks of 256 threads per SM)
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long maxb = (P->M + chunk - 1) / chunk;
  return (int)std::max(1LL, std::min<long long>(maxb, (long long)P->sms * 8 / nb));
}

inline fm_status ensure_reduce(fm_plan* P, int nb, int K) {
  const int nblk = red_blocks_max(P, nb);
  FM_CK(P->red_part.ensure((size_t)nb * nblk * (KV_KMAX + 2) * sizeof(double2)));
  FM_CK(P->red_out.ensure((size_t)nb * (KV_KMAX + 2) * sizeof(double2)));
  if (P->red_cnt.cap < (size_t)nb * sizeof(unsigned)) {
    FM_CK(P->red_cnt.ensure((size_t)nb * sizeof(unsigned)));
    FM_CK(cudaMemsetAsync(P->red_cnt.p, 0, (size_t)nb * sizeof(unsigned), P->st));
  }
  (void)K;
  return FM_OK;
}

// Per-RHS operator data for batches whose right-hand sides do not share one potential
// (the slot engine): potentials at V + b*vstride, per-RHS eps_imag, and per-RHS input/output vectors.
struct RhsCtx {
  const void* V = nullptr;
  long long vstride = 0;
  const double* ksq_im_b = nullptr;   // eps_imag / k_ref^2 per RHS
  const double* inv_eps_b = nullptr;  // k_ref^2 / eps_imag per RHS
  VecTab vt;
};

// ---- operator drivers (fm_ops.cu) ----
// Green application / CBS operator on device buffers (plan precision): in -> out (nb fields; out may not alias
// in, t1, t2); pro: PRO_COPY, PRO_V or PRO_V_SCALE applied to `in`; epi: EPI_* applied to g = G_avg(psi).
// chain (applications in sequence, each on the previous one's output; only where green_chain_ok):
//   GREEN_CHAIN_HAVE_XF   t1 already holds the x pass of PRO_V on `in` (the previous call left it): skip it
//   GREEN_CHAIN_NEXT_XF   EPI_PREC_OP whose XI pass also leaves the x pass of PRO_V on `out` in t1
enum { GREEN_CHAIN_HAVE_XF = 1, GREEN_CHAIN_NEXT_XF = 2 };
template <typename R>
fm_status green_op(fm_plan* P, int nb, const void* in, int pro, const double* rs, int epi, const void* xv,
                   const void* bv, const EpiParams& ep_in, void* out, const int* act, int nact = -1,
                   const RhsCtx* rc = nullptr, int chain = 0);
// the five fused passes (no shift, or z-only shifts in one length-2L z pass), contiguous batches: where green_op
// can chain applications
inline bool green_chain_ok(const fm_plan* P, const RhsCtx* rc) {
  return !P->generic && (!P->avg || P->zonly) && !(rc && (rc->vt.in || rc->vt.out));
}
// H = -i lambda/(2 pi 377) curl(E) for nb fields (in -> out, contiguous batches; act masks RHS)
template <typename R>
fm_status curl_batch(fm_plan* P, int nb, const void* in, void* out, const int* act);

// ---- Krylov drivers (fm_gmres.cu) ----
template <typename R>
fm_status multidot(fm_plan* P, int nb, int K, const void* U, const void* w, bool wnorm, const int* act,
                   std::vector<double2>& host_out, int nact = -1);
template <typename R>
fm_status axpby3(fm_plan* P, int nb, const void* a, const std::vector<cd>& ca, const void* b,
                 const std::vector<cd>& cbv, const void* c, const std::vector<cd>& ccv, void* y, bool norm,
                 const int* act, std::vector<double>* norms);
void sym_givens(cd a, double b, double& c, cd& s, cd& rho);
// Block Gram-Schmidt kernels on the FP64 tensor cores.  which: 0 block dot D = X^H Y, 1 block update into the
// basis, 2 block update in place into Y, 3 orthonormalisation V = Z Rb^{-1}.  Kb (optional, device): per-RHS
// basis sizes <= K for 0-2, and for 3 the per-RHS first basis row of the output (Z then points at row 0).
template <typename R, typename YR>
cudaError_t block_kernels(fm_plan* P, int which, int S, int nb, int K, const void* U, const void* Y, void* Z,
                          const int* act, int nact, const int* Kb = nullptr);
// vectors per block of block GMRES (fm_solve_opts.block; 0 selects 4)
inline int block_size_of(const fm_solve_opts& o) { return o.block > 0 ? o.block : 4; }
double now_s();
fm_status check_device_error(fm_plan* P);
// from scaled source terms in P->sbuf (nb RHS) to the scattered field in P->xbuf and its curl in P->ebuf
template <typename R>
fm_status solve_core(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info);

// ---- plane-wave tables and scalars (fm_capi.cu) ----
void set_scalars(fm_plan* P, double k_bg, double eps_imag, double wavelength);
fm_status wave_tables(const fm_plan* P, const fm_plane_wave& w, double eps_bg, double2* tx, double2* ty,
                      double2* tz, double2* pe, double2* ph);
