// libfmcuda: plan object, CBS operator drivers, Krylov drivers and the C ABI.
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

static thread_local std::string g_err;

namespace fm {
// lets other translation units of the library report through fm_last_error()
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace fm

static fm_status fail(fm_status s, const std::string& msg) {
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

namespace {

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

}  // namespace

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
static const char* kcls_name[KC_N] = {"xf", "yf", "zg", "yi", "xi", "multidot", "update", "mgs/gram", "axpby", "curl", "setup"};

static cudaEvent_t ev_get(fm_plan* P) {
  if (!P->evpool.empty()) {
    cudaEvent_t e = P->evpool.back();
    P->evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

static void tk_resolve(fm_plan* P) {
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
static Tk tk_begin(fm_plan* P, int cls, double bytes) {
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
static void tk_end(const Tk& t) {
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
static int red_blocks_max(const fm_plan* P, int nb) {
  // upper bound of kv_blocks over all kernels (at most 8 blocks of 256 threads per SM)
  const long long chunk = (long long)KV_THREADS * KV_EPT;
  const long long maxb = (P->M + chunk - 1) / chunk;
  return (int)std::max(1LL, std::min<long long>(maxb, (long long)P->sms * 8 / nb));
}

static fm_status ensure_reduce(fm_plan* P, int nb, int K) {
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

// ---------------------------------------------------------------------------
// Green application / CBS operator on device buffers (plan precision)
//   in  : nb fields
//   out : nb fields (may not alias in, t1, t2)
//   pro : PRO_COPY (psi = in) or PRO_V / PRO_V_SCALE (psi = V.*in [* scale])
//   epi : EPI_* epilogue applied to g = G_avg(psi)
// ---------------------------------------------------------------------------
// Per-RHS operator data for batches whose right-hand sides do not share one potential
// (the slot engine): potentials at V + b*vstride, per-RHS eps_imag, and per-RHS input/output vectors.
struct RhsCtx {
  const void* V = nullptr;
  long long vstride = 0;
  const double* ksq_im_b = nullptr;   // eps_imag / k_ref^2 per RHS
  const double* inv_eps_b = nullptr;  // k_ref^2 / eps_imag per RHS
  VecTab vt;
};

// ---------------------------------------------------------------------------
// General-length path (fm_generic.cuh): plain passes, one or two branches
// ---------------------------------------------------------------------------
template <typename S>
static cudaError_t gen_axis(const fm_plan* P, const Dims& d, int axis, int dir, void* f, const int* act) {
  if constexpr (std::is_same<S, double>::value)
    return launch_gen_axis<double, double>(d, axis, dir, f, f, P->gax[axis], act, P->st);
  else return P->c64 ? launch_gen_axis<float, double>(d, axis, dir, f, f, P->gax[axis], act, P->st)
                     : launch_gen_axis<float, float>(d, axis, dir, f, f, P->gax[axis], act, P->st);
}
template <typename S>
static cudaError_t gen_pre(const fm_plan* P, const Dims& d, int pro, const void* in, const void* V, const double* rs,
                           const GenRamps& rp, void* out, const int* act, VecTab vt) {
  if constexpr (std::is_same<S, double>::value)
    return launch_gen_pre<double, double>(d, pro, in, V, rs, rp, out, act, P->st, vt);
  else return P->c64 ? launch_gen_pre<float, double>(d, pro, in, V, rs, rp, out, act, P->st, vt)
                     : launch_gen_pre<float, float>(d, pro, in, V, rs, rp, out, act, P->st, vt);
}
template <typename S>
static cudaError_t gen_kspace(const fm_plan* P, const Dims& d, int mode, void* f, const GreenParams& gp, const int* act) {
  if constexpr (std::is_same<S, double>::value) return launch_gen_kspace<double, double>(d, mode, f, gp, act, P->st);
  else return P->c64 ? launch_gen_kspace<float, double>(d, mode, f, gp, act, P->st)
                     : launch_gen_kspace<float, float>(d, mode, f, gp, act, P->st);
}
template <typename S>
static cudaError_t gen_post(const fm_plan* P, const Dims& d, int epi, const void* in, const void* V, const void* xv,
                            const void* bv, const double* rs, const EpiParams& ep, const GenRamps& rp, void* out,
                            const int* act, VecTab vt) {
  if constexpr (std::is_same<S, double>::value)
    return launch_gen_post<double, double>(d, epi, in, V, xv, bv, rs, ep, rp, out, act, P->st, vt);
  else return P->c64 ? launch_gen_post<float, double>(d, epi, in, V, xv, bv, rs, ep, rp, out, act, P->st, vt)
                     : launch_gen_post<float, float>(d, epi, in, V, xv, bv, rs, ep, rp, out, act, P->st, vt);
}

// The Green application / CBS operator of green_op on a plan with an axis that has no fused pass.  Per branch:
// PRE (potential, forward ramps) -> forward DFT along x, y, z -> Green of the branch -> inverse DFT along z, y,
// x -> POST (reverse ramps, epilogue).  With an absorbing axis the +s branch stores half its result in t3 and
// the -s branch adds it before the epilogue (dyadic_green.jl:127-152).
template <typename R>
static fm_status gen_green_op(fm_plan* P, int nb, const void* in, int pro, const double* rs, int epi, const void* xv,
                              const void* bv, const EpiParams& ep_in, void* out, const int* act, int nact,
                              const RhsCtx* rc) {
  using T = cplx<R>;
  if (nact < 0) nact = nb;
  EpiParams ep = ep_in;
  if (rc) ep.inv_eps_b = rc->inv_eps_b;
  Dims d = P->dims;
  d.nb = nb;
  const size_t fbytes = (size_t)nb * P->M * sizeof(T);
  const double fbA = (double)nact * P->M * sizeof(T), vb = (double)nact * P->n * sizeof(T);
  FM_CK(P->t1.ensure(fbytes));
  const int nbr = P->avg ? 2 : 1;
  if (nbr == 2) FM_CK(P->t3.ensure(fbytes));
  GreenParams gp{};
  const double kr = std::sqrt(P->kref2);
  for (int a = 0; a < 3; ++a) gp.dk[a] = 2.0 * M_PI / ((double)(a == 0 ? d.nx : a == 1 ? d.ny : d.nz) * P->desc.resolution[a]) / kr;
  gp.ksq_re = P->k_bg * P->k_bg / P->kref2;
  gp.ksq_im = P->eps_imag / P->kref2;
  gp.scale_re = 1.0 / ((double)P->n * nbr);
  const void* V = P->V.p;
  VecTab vt{};
  if (rc) {
    V = rc->V;
    d.vstride = rc->vstride;
    gp.ksq_im_b = rc->ksq_im_b;
    vt = rc->vt;
  }
  double postb = 2 * fbA;
  if (epi != EPI_STORE) postb += fbA;
  if (epi == EPI_PREC_RES) postb += fbA;
  if (epi == EPI_PREC_OP || epi == EPI_PREC_RES) postb += vb;
  if (epi == EPI_OP && (ep.beta_re != 0.0 || ep.beta_im != 0.0)) postb += fbA;
  const DevBuf* rpos[3] = {&P->rxp, &P->ryp, &P->rzp};
  const DevBuf* rneg[3] = {&P->rxm, &P->rym, &P->rzm};
  cudaError_t e;
  for (int br = 0; br < nbr; ++br) {
    GenRamps rp;
    for (int a = 0; a < 3; ++a) {
      gp.shift[a] = (br == 0 ? 1.0 : -1.0) * P->shift[a];
      rp.r[a] = P->shift[a] != 0.0 ? (br == 0 ? rpos[a]->p : rneg[a]->p) : nullptr;
    }
    FM_TRACK(P, KC_XF, 2 * fbA + (pro != PRO_COPY ? vb : 0.0),
             e = gen_pre<R>(P, d, pro, in, V, rs, rp, P->t1.p, act, vt));
    FM_CK(e);
    for (int a = 0; a < 3; ++a) {
      FM_TRACK(P, KC_YF, 2 * fbA, e = gen_axis<R>(P, d, a, -1, P->t1.p, act));
      FM_CK(e);
    }
    FM_TRACK(P, KC_ZG, 2 * fbA, e = gen_kspace<R>(P, d, ZMODE_ONE, P->t1.p, gp, act));
    FM_CK(e);
    for (int a = 2; a >= 0; --a) {
      FM_TRACK(P, KC_YI, 2 * fbA, e = gen_axis<R>(P, d, a, +1, P->t1.p, act));
      FM_CK(e);
    }
    if (nbr == 2 && br == 0) {
      EpiParams e0{};
      FM_TRACK(P, KC_XI, 2 * fbA,
               e = gen_post<R>(P, d, EPI_STORE, P->t1.p, V, nullptr, nullptr, nullptr, e0, rp, P->t3.p, act, VecTab{}));
    } else {
      EpiParams e1 = ep;
      if (nbr == 2) e1.gadd = P->t3.p;
      FM_TRACK(P, KC_XI, postb + (nbr == 2 ? fbA : 0.0),
               e = gen_post<R>(P, d, epi, P->t1.p, V, xv, bv, rs, e1, rp, out, act, vt));
    }
    FM_CK(e);
  }
  return FM_OK;
}

template <typename R>
static fm_status green_op(fm_plan* P, int nb, const void* in, int pro, const double* rs, int epi, const void* xv,
                          const void* bv, const EpiParams& ep_in, void* out, const int* act, int nact = -1,
                          const RhsCtx* rc = nullptr) {
  using T = cplx<R>;
  if (P->generic) return gen_green_op<R>(P, nb, in, pro, rs, epi, xv, bv, ep_in, out, act, nact, rc);
  if (nact < 0) nact = nb;
  EpiParams ep = ep_in;
  if (rc) ep.inv_eps_b = rc->inv_eps_b;
  const double fbA = (double)nact * P->M * sizeof(T), vb = (double)nact * P->n * sizeof(T);
  double xib = 2 * fbA;
  if (epi != EPI_STORE) xib += fbA;
  if (epi == EPI_PREC_RES) xib += fbA;
  if (epi == EPI_PREC_OP || epi == EPI_PREC_RES) xib += vb;
  if (epi == EPI_OP && (ep.beta_re != 0.0 || ep.beta_im != 0.0)) xib += fbA;
  Dims d = P->dims;
  d.nb = nb;
  const size_t fbytes = (size_t)nb * P->M * sizeof(T);
  FM_CK(P->t1.ensure(fbytes));
  FM_CK(P->t2.ensure(fbytes));
  GreenParams gp{};
  const double kr = std::sqrt(P->kref2);
  for (int a = 0; a < 3; ++a) gp.dk[a] = 2.0 * M_PI / ((double)(a == 0 ? d.nx : a == 1 ? d.ny : d.nz) * P->desc.resolution[a]) / kr;
  gp.ksq_re = P->k_bg * P->k_bg / P->kref2;
  gp.ksq_im = P->eps_imag / P->kref2;
  const void* V = P->V.p;
  VecTab vt{};
  if (rc) {
    V = rc->V;
    d.vstride = rc->vstride;
    gp.ksq_im_b = rc->ksq_im_b;
    vt = rc->vt;
  }
  if (!P->avg || P->zonly) {
    const int mode = P->zonly ? ZMODE_AVG2 : ZMODE_ONE;
    gp.shift[2] = P->zonly ? P->shift[2] : 0.0;
    gp.scale_re = 1.0 / ((double)P->n * (P->zonly ? 2.0 : 1.0));
    cudaError_t e;
    FM_TRACK(P, KC_XF, 2 * fbA + (pro != PRO_COPY ? vb : 0.0),
             e = pass_xf<R>(P, d, pro, in, V, rs, P->twx.p, nullptr, P->t1.p, act, vt));
    FM_CK(e);
    FM_TRACK(P, KC_YF, 2 * fbA, e = pass_y<R>(P, d, -1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_ZG, 2 * fbA,
             e = pass_zg<R>(P, d, mode, P->t2.p, gp, P->zonly ? P->twz2.p : P->twz.p, P->zonly ? P->rz.p : nullptr,
                              P->t1.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_YI, 2 * fbA, e = pass_y<R>(P, d, +1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_XI, xib, e = pass_xi<R>(P, d, epi, P->t2.p, V, xv, bv, rs, ep, P->twx.p, nullptr, out, act, vt));
    FM_CK(e);
    return FM_OK;
  }
  if (P->zsplit) {
    // the two z branches (+s, -s) as two length-L z passes with their phase ramps; the second adds to the first
    gp.scale_re = 1.0 / ((double)P->n * 2.0);
    cudaError_t e;
    FM_TRACK(P, KC_XF, 2 * fbA + (pro != PRO_COPY ? vb : 0.0),
             e = pass_xf<R>(P, d, pro, in, V, rs, P->twx.p, nullptr, P->t1.p, act, vt));
    FM_CK(e);
    FM_TRACK(P, KC_YF, 2 * fbA, e = pass_y<R>(P, d, -1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
    FM_CK(e);
    gp.shift[2] = P->shift[2];
    gp.accumulate = 0;
    FM_TRACK(P, KC_ZG, 2 * fbA, e = pass_zg<R>(P, d, ZMODE_ONE, P->t2.p, gp, P->twz.p, P->rzp.p, P->t1.p, act));
    FM_CK(e);
    gp.shift[2] = -P->shift[2];
    gp.accumulate = 1;
    FM_TRACK(P, KC_ZG, 3 * fbA, e = pass_zg<R>(P, d, ZMODE_ONE, P->t2.p, gp, P->twz.p, P->rzm.p, P->t1.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_YI, 2 * fbA, e = pass_y<R>(P, d, +1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_XI, xib, e = pass_xi<R>(P, d, epi, P->t2.p, V, xv, bv, rs, ep, P->twx.p, nullptr, out, act, vt));
    FM_CK(e);
    return FM_OK;
  }
  // General case: sub-pixel shifts on x or y (absorbing x or y boundaries).  The branches G(+s) and G(-s)
  // (dyadic_green.jl:127-152) differ on every shifted axis, so each runs its own five passes with its phase
  // ramps (dyadic_green.jl:243-266, per axis: x in the x passes, y in the y passes, z in the z pass) and its
  // shifted k (dyadic_green.jl:189-221).  Branch + stores half of G(+s) psi in t3; branch - adds it to half of
  // G(-s) psi in the XI pass, before the epilogue.
  {
    FM_CK(P->t3.ensure(fbytes));
    gp.scale_re = 1.0 / ((double)P->n * 2.0);
    cudaError_t e;
    for (int br = 0; br < 2; ++br) {
      const double sg = br == 0 ? 1.0 : -1.0;
      for (int a = 0; a < 3; ++a) gp.shift[a] = sg * P->shift[a];
      const void* rx = P->shift[0] != 0.0 ? (br == 0 ? P->rxp.p : P->rxm.p) : nullptr;
      const void* ry = P->shift[1] != 0.0 ? (br == 0 ? P->ryp.p : P->rym.p) : nullptr;
      const void* rzt = P->shift[2] != 0.0 ? (br == 0 ? P->rzp.p : P->rzm.p) : nullptr;
      FM_TRACK(P, KC_XF, 2 * fbA + (pro != PRO_COPY ? vb : 0.0),
               e = pass_xf<R>(P, d, pro, in, V, rs, P->twx.p, rx, P->t1.p, act, vt));
      FM_CK(e);
      FM_TRACK(P, KC_YF, 2 * fbA, e = pass_y<R>(P, d, -1, P->t1.p, P->twy.p, ry, P->t2.p, act));
      FM_CK(e);
      FM_TRACK(P, KC_ZG, 2 * fbA, e = pass_zg<R>(P, d, ZMODE_ONE, P->t2.p, gp, P->twz.p, rzt, P->t1.p, act));
      FM_CK(e);
      FM_TRACK(P, KC_YI, 2 * fbA, e = pass_y<R>(P, d, +1, P->t1.p, P->twy.p, ry, P->t2.p, act));
      FM_CK(e);
      if (br == 0) {
        EpiParams e0{};
        FM_TRACK(P, KC_XI, 2 * fbA,
                 e = pass_xi<R>(P, d, EPI_STORE, P->t2.p, V, nullptr, nullptr, nullptr, e0, P->twx.p, rx, P->t3.p,
                                act));
      } else {
        EpiParams e1 = ep;
        e1.gadd = P->t3.p;
        FM_TRACK(P, KC_XI, xib + fbA,
                 e = pass_xi<R>(P, d, epi, P->t2.p, V, xv, bv, rs, e1, P->twx.p, rx, out, act, vt));
      }
      FM_CK(e);
    }
    return FM_OK;
  }
}

// ---------------------------------------------------------------------------
// Krylov helpers
// ---------------------------------------------------------------------------
template <typename R>
static fm_status multidot(fm_plan* P, int nb, int K, const void* U, const void* w, bool wnorm, const int* act,
                          std::vector<double2>& host_out, int nact = -1) {
  FM_TRY(ensure_reduce(P, nb, K));
  if (nact < 0) nact = nb;
  const int nblk = wnorm ? kv_blocks(P, k_multidot<R, true>, nb) : kv_blocks(P, k_multidot<R, false>, nb);
  dim3 g(nblk, nb);
  const double bytes = (double)(K + 1) * nact * P->M * sizeof(cplx<R>);
  if (wnorm)
    FM_TRACK(P, KC_DOT, bytes,
             (k_multidot<R, true><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, K, (const cplx<R>*)U, (const cplx<R>*)w,
                                                               (double2*)P->red_part.p, (double2*)P->red_out.p,
                                                               (unsigned*)P->red_cnt.p, act)));
  else
    FM_TRACK(P, KC_DOT, bytes,
             (k_multidot<R, false><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, K, (const cplx<R>*)U, (const cplx<R>*)w,
                                                                (double2*)P->red_part.p, (double2*)P->red_out.p,
                                                                (unsigned*)P->red_cnt.p, act)));
  FM_CK(cudaGetLastError());
  const int KK = K + (wnorm ? 1 : 0);
  host_out.resize((size_t)nb * KK);
  FM_CK(cudaMemcpyAsync(host_out.data(), P->red_out.p, host_out.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  tk_resolve(P);
  return FM_OK;
}

// y = ca*a + cb*b + cc*c per RHS (host coefficient vectors of length nb, empty -> operand skipped)
template <typename R>
static fm_status axpby3(fm_plan* P, int nb, const void* a, const std::vector<cd>& ca, const void* b,
                        const std::vector<cd>& cb, const void* c, const std::vector<cd>& cc, void* y, bool norm,
                        const int* act, std::vector<double>* nrm) {
  FM_TRY(ensure_reduce(P, nb, 1));
  FM_CK(P->coef.ensure((size_t)3 * nb * sizeof(double2)));
  std::vector<double2> h((size_t)3 * nb, make_double2(0, 0));
  for (int i = 0; i < nb; ++i) {
    if (a) h[i] = make_double2(ca[i].real(), ca[i].imag());
    if (b) h[nb + i] = make_double2(cb[i].real(), cb[i].imag());
    if (c) h[2 * nb + i] = make_double2(cc[i].real(), cc[i].imag());
  }
  FM_CK(cudaMemcpyAsync(P->coef.p, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
  const double2* cp = (const double2*)P->coef.p;
  const int nblk = norm ? kv_blocks(P, k_axpby3<R, true>, nb) : kv_blocks(P, k_axpby3<R, false>, nb);
  dim3 g(nblk, nb);
  using T = cplx<R>;
  const double bytes = (double)((a ? 1 : 0) + (b ? 1 : 0) + (c ? 1 : 0) + 1) * nb * P->M * sizeof(T);
  if (norm)
    FM_TRACK(P, KC_AXPBY, bytes,
             (k_axpby3<R, true><<<g, KV_THREADS, 0, P->st>>>(P->M, (const T*)a, cp, (const T*)b, cp + nb, (const T*)c,
                                                             cp + 2 * nb, (T*)y, (double2*)P->red_part.p,
                                                             (double2*)P->red_out.p, (unsigned*)P->red_cnt.p, act)));
  else
    FM_TRACK(P, KC_AXPBY, bytes,
             (k_axpby3<R, false><<<g, KV_THREADS, 0, P->st>>>(P->M, (const T*)a, cp, (const T*)b, cp + nb, (const T*)c,
                                                              cp + 2 * nb, (T*)y, nullptr, nullptr, nullptr, act)));
  FM_CK(cudaGetLastError());
  if (norm) {
    std::vector<double2> o(nb);
    FM_CK(cudaMemcpyAsync(o.data(), P->red_out.p, nb * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
    tk_resolve(P);
    nrm->resize(nb);
    for (int i = 0; i < nb; ++i) (*nrm)[i] = o[i].x;
  }
  return FM_OK;
}

static void sym_givens(cd a, double b, double& c, cd& s, cd& rho) {
  const double aa = std::abs(a);
  if (b == 0.0) {
    c = 1.0;
    s = 0.0;
    rho = a;
  } else if (aa == 0.0) {
    c = 0.0;
    s = 1.0;
    rho = b;
  } else {
    const double r = std::hypot(aa, b);
    c = aa / r;
    s = (a / aa) * (b / r);
    rho = (a / aa) * r;
  }
}

struct RhsState {
  bool active = true;
  bool solved = false;
  int iters = 0;
  double beta = 0, eps = 0, rnorm = 0;
  std::vector<double> c;
  std::vector<cd> s, z;
  std::vector<std::vector<cd>> R;  // columns
  int inner = 0;
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// GMRES (Krylov.jl semantics) on a batch of nb RHS; b in P->bbuf, x (warm
// start u0 = b) in P->xbuf.  Basis vectors are kept unnormalised with their
// scale 1/h_{k+1,k} in P->scale (deferred normalisation).
// ---------------------------------------------------------------------------
template <typename R>
static fm_status gmres(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info, double deadline) {
  using T = cplx<R>;
  const size_t fe = (size_t)P->M;
  const size_t fbytes = (size_t)nb * fe * sizeof(T);
  const int itmax = std::max(1, o.maxiters);
  const int mem = (o.restart > 0) ? std::min(o.restart, itmax) : itmax;
  if (mem + 1 > KV_KMAX) return fail(FM_ERR_UNSUPPORTED, "Krylov basis larger than 127 vectors");
  FM_CK(P->basis.ensure((size_t)(mem + 1) * fbytes));
  FM_CK(P->scale.ensure((size_t)(KV_KMAX + 1) * nb * sizeof(double)));
  FM_CK(P->hbuf.ensure((size_t)nb * (KV_KMAX + 2) * sizeof(double2)));
  FM_CK(P->active.ensure((size_t)nb * sizeof(int)));
  FM_TRY(ensure_reduce(P, nb, mem + 1));
  T* U = (T*)P->basis.p;
  double* sc = (double*)P->scale.p;
  int* act = (int*)P->active.p;
  const double btol = std::pow(2.220446049250313e-16, 0.75);

  std::vector<RhsState> S(nb);
  std::vector<int> acth(nb, 1);
  std::vector<double> sch((size_t)(KV_KMAX + 1) * nb, 0.0);
  EpiParams ep{};
  ep.inv_eps = P->kref2 / P->eps_imag;
  auto upload_active = [&]() -> fm_status {
    FM_CK(cudaMemcpyAsync(act, acth.data(), nb * sizeof(int), cudaMemcpyHostToDevice, P->st));
    return FM_OK;
  };
  auto upload_scale_col = [&](int j) -> fm_status {
    FM_CK(cudaMemcpyAsync(sc + (size_t)j * nb, sch.data() + (size_t)j * nb, nb * sizeof(double), cudaMemcpyHostToDevice,
                          P->st));
    return FM_OK;
  };
  // r0 = M^{-1}(b - A x) into U[0]
  auto residual_into_U0 = [&](const int* a) -> fm_status {
    return green_op<R>(P, nb, P->xbuf.p, PRO_V, nullptr, EPI_PREC_RES, P->xbuf.p, P->bbuf.p, ep, U, a);
  };

  FM_TRY(upload_active());
  FM_TRY(residual_into_U0(act));
  std::vector<double2> hv;
  FM_TRY(multidot<R>(P, nb, 0, U, U, true, act, hv));
  int iter = 0;
  for (int b = 0; b < nb; ++b) {
    S[b].beta = std::sqrt(hv[b].x);
    S[b].rnorm = S[b].beta;
    S[b].eps = o.abstol + o.reltol * S[b].beta;
    info[b].residual0 = S[b].beta;
    if (S[b].beta == 0.0) {
      S[b].active = false;
      S[b].solved = true;
      acth[b] = 0;
    } else if (S[b].rnorm <= S[b].eps) {
      S[b].active = false;
      S[b].solved = true;
      acth[b] = 0;
    }
  }
  bool any = false;
  for (int b = 0; b < nb; ++b) any |= S[b].active;
  std::vector<int> started(nb, 0);
  while (any && iter < itmax) {
    // (re)start: U[0] = r0 (already for the first pass), z[0] = beta
    for (int b = 0; b < nb; ++b) {
      if (!S[b].active) continue;
      S[b].c.clear(); S[b].s.clear(); S[b].R.clear(); S[b].z.assign(1, cd(S[b].beta, 0)); S[b].inner = 0;
      sch[b] = 1.0 / S[b].beta;
    }
    FM_TRY(upload_active());
    FM_TRY(upload_scale_col(0));
    int j = 0;
    bool pass_done = false;
    while (!pass_done) {
      // w = M^{-1} A v_j  into U[j+1]
      T* Uj = U + (size_t)j * nb * fe;
      T* Uw = U + (size_t)(j + 1) * nb * fe;
      int nact = 0;
      for (int b = 0; b < nb; ++b) nact += acth[b];
      const double fbA = (double)nact * fe * sizeof(T);
      FM_TRY(green_op<R>(P, nb, Uj, PRO_V_SCALE, sc + (size_t)j * nb, EPI_PREC_OP, Uj, nullptr, ep, Uw, act, nact));
      // orthogonalise against v_0..v_j
      const int K = j + 1;
      std::vector<double2> hcol((size_t)nb * (K + 1));
      if (o.ortho == FM_ORTHO_MGS) {
        double2* hd = (double2*)P->hbuf.p;
        const int hs = KV_KMAX + 2;
        dim3 g(kv_blocks(P, k_mgs<R>, nb), nb);
        for (int i = 0; i <= K; ++i) {
          const double mb = fbA * ((i > 0 ? 1 : 0) + (i < K ? 1 : 0) + 1 + (i > 0 ? 1 : 0));
          FM_TRACK(P, KC_MGS, mb,
                   (k_mgs<R><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, i, K, U, sc, nb, Uw, hd, hs,
                                                          (double2*)P->red_part.p, (unsigned*)P->red_cnt.p, act)));
        }
        FM_CK(cudaGetLastError());
        std::vector<double2> hh((size_t)nb * hs);
        FM_CK(cudaMemcpyAsync(hh.data(), hd, hh.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
        FM_CK(cudaStreamSynchronize(P->st));
        tk_resolve(P);
        for (int b = 0; b < nb; ++b)
          for (int i = 0; i <= K; ++i) hcol[(size_t)b * (K + 1) + i] = hh[(size_t)b * hs + i];
      } else {
        // classical Gram-Schmidt (optionally twice), FP64 coefficients
        std::vector<double2> hr;
        FM_TRY(multidot<R>(P, nb, K, U, Uw, false, act, hr, nact));
        std::vector<double2> htot((size_t)nb * K);
        for (int b = 0; b < nb; ++b)
          for (int i = 0; i < K; ++i) {
            double s = sch[(size_t)i * nb + b];
            htot[(size_t)b * K + i] = make_double2(hr[(size_t)b * K + i].x * s, hr[(size_t)b * K + i].y * s);
          }
        const int passes = (o.ortho == FM_ORTHO_CGS2) ? 2 : 1;
        for (int pass = 0; pass < passes; ++pass) {
          const bool last = (pass == passes - 1);
          // raw projections <U_i, w>; the update coefficient of U_i is sc_i^2 * hr_i
          FM_CK(P->coef.ensure((size_t)nb * K * sizeof(double2)));
          FM_CK(cudaMemcpyAsync(P->coef.p, hr.data(), hr.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
          Coef cf{(const double2*)P->coef.p, K, sc, nb, -1.0, 0};
          const double ub = (K + 2) * fbA;
          dim3 g(last ? kv_blocks(P, k_update<R, true>, nb) : kv_blocks(P, k_update<R, false>, nb), nb);
          if (last)
            FM_TRACK(P, KC_UPD, ub,
                     (k_update<R, true><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, K, U, cf, Uw, nullptr,
                                                                     (double2*)P->red_part.p, (double2*)P->red_out.p,
                                                                     (unsigned*)P->red_cnt.p, act)));
          else
            FM_TRACK(P, KC_UPD, ub,
                     (k_update<R, false><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, K, U, cf, Uw, nullptr, nullptr, nullptr,
                                                                      nullptr, act)));
          FM_CK(cudaGetLastError());
          if (!last) {
            FM_TRY(multidot<R>(P, nb, K, U, Uw, false, act, hr, nact));
            for (int b = 0; b < nb; ++b)
              for (int i = 0; i < K; ++i) {
                double s = sch[(size_t)i * nb + b];
                htot[(size_t)b * K + i].x += hr[(size_t)b * K + i].x * s;
                htot[(size_t)b * K + i].y += hr[(size_t)b * K + i].y * s;
              }
          }
        }
        std::vector<double2> nn(nb);
        FM_CK(cudaMemcpyAsync(nn.data(), P->red_out.p, nb * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
        FM_CK(cudaStreamSynchronize(P->st));
        tk_resolve(P);
        for (int b = 0; b < nb; ++b) {
          for (int i = 0; i < K; ++i) hcol[(size_t)b * (K + 1) + i] = htot[(size_t)b * K + i];
          hcol[(size_t)b * (K + 1) + K] = nn[b];
        }
      }
      ++iter;
      // Givens update per RHS
      bool any_left = false;
      for (int b = 0; b < nb; ++b) {
        RhsState& r = S[b];
        if (!r.active) continue;
        std::vector<cd> col(K);
        for (int i = 0; i < K; ++i) col[i] = cd(hcol[(size_t)b * (K + 1) + i].x, hcol[(size_t)b * (K + 1) + i].y);
        const double hb = std::sqrt(std::max(0.0, hcol[(size_t)b * (K + 1) + K].x));
        for (int i = 0; i < K - 1; ++i) {
          cd t = r.c[i] * col[i] + r.s[i] * col[i + 1];
          col[i + 1] = std::conj(r.s[i]) * col[i] - r.c[i] * col[i + 1];
          col[i] = t;
        }
        double c;
        cd s, rho;
        sym_givens(col[K - 1], hb, c, s, rho);
        col[K - 1] = rho;
        r.c.push_back(c);
        r.s.push_back(s);
        r.R.push_back(col);
        const cd zk1 = std::conj(s) * r.z[K - 1];
        r.z[K - 1] = c * r.z[K - 1];
        r.rnorm = std::abs(zk1);
        r.inner = K;
        r.iters += 1;
        const bool solved = (r.rnorm <= r.eps) || (r.rnorm + 1.0 <= 1.0);
        const bool breakdown = hb <= btol;
        const bool tired = iter >= itmax;
        const bool inner_tired = K >= mem;
        r.solved = solved;
        if (solved || breakdown || tired || inner_tired) {
          acth[b] = 0;  // this pass is over for b
          if (solved || breakdown || tired) r.active = false;
        } else {
          r.z.push_back(zk1);
          sch[(size_t)(j + 1) * nb + b] = 1.0 / hb;
          any_left = true;
        }
        if (breakdown) r.active = false;
      }
      if (deadline > 0 && now_s() > deadline) return fail(FM_ERR_TIMEOUT, "solve deadline passed");
      if (!any_left) {
        pass_done = true;
      } else {
        FM_TRY(upload_active());
        FM_TRY(upload_scale_col(j + 1));
        ++j;
      }
    }
    // x += sum_i y_i v_i  per RHS that took part in this pass
    std::vector<double2> yh((size_t)nb * (KV_KMAX + 1), make_double2(0, 0));
    int Kmax = 0;
    for (int b = 0; b < nb; ++b) {
      RhsState& r = S[b];
      const int n_in = r.inner;
      if (n_in == 0) continue;
      std::vector<cd> y(r.z.begin(), r.z.begin() + n_in);
      for (int i = n_in - 1; i >= 0; --i) {
        for (int jj = n_in - 1; jj > i; --jj) y[i] -= r.R[jj][i] * y[jj];
        if (std::abs(r.R[i][i]) <= btol) {
          for (int q = 0; q <= i; ++q) y[q] = 0.0;
          break;
        }
        y[i] /= r.R[i][i];
      }
      for (int i = 0; i < n_in; ++i) yh[(size_t)b * (KV_KMAX + 1) + i] = make_double2(y[i].real(), y[i].imag());
      Kmax = std::max(Kmax, n_in);
      r.inner = 0;
    }
    if (Kmax > 0) {
      FM_CK(P->coef.ensure(yh.size() * sizeof(double2)));
      FM_CK(cudaMemcpyAsync(P->coef.p, yh.data(), yh.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync(sc, sch.data(), (size_t)(KV_KMAX + 1) * nb * sizeof(double), cudaMemcpyHostToDevice, P->st));
      Coef cf{(const double2*)P->coef.p, KV_KMAX + 1, sc, nb, 1.0, 1};
      dim3 g(kv_blocks(P, k_update<R, false>, nb), nb);
      FM_TRACK(P, KC_UPD, (double)(Kmax + 2) * nb * fe * sizeof(T),
               (k_update<R, false><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, Kmax, U, cf, (T*)P->xbuf.p, nullptr, nullptr,
                                                                nullptr, nullptr, nullptr)));
      FM_CK(cudaGetLastError());
    }
    any = false;
    for (int b = 0; b < nb; ++b) {
      acth[b] = S[b].active ? 1 : 0;
      any |= S[b].active;
    }
    if (any && iter < itmax) {
      // restart: new residual for the RHS still running
      FM_TRY(upload_active());
      FM_TRY(residual_into_U0(act));
      FM_TRY(multidot<R>(P, nb, 0, U, U, true, act, hv));
      for (int b = 0; b < nb; ++b)
        if (S[b].active) S[b].beta = std::sqrt(hv[b].x);
    }
  }
  for (int b = 0; b < nb; ++b) {
    info[b].iterations = S[b].iters;
    info[b].solved = S[b].solved ? 1 : 0;
    info[b].residual = S[b].rnorm;
  }
  return FM_OK;
}

// ---------------------------------------------------------------------------
// s-step (block) GMRES
//
// The stored basis is a sequence of raw vectors X_0..X_K-1 in U; the
// orthonormal Arnoldi basis is V = X Rf^{-1}, with Rf upper triangular and
// block diagonal (1x1 blocks for the classical Gram-Schmidt steps, S x S
// blocks for each s-step block), held per RHS on the host in FP64.  Every
// coefficient that touches the basis is transformed on the host, so the
// device only sees raw combinations of stored vectors.
//
// After S classical Gram-Schmidt steps (which also give Ritz values for the
// first Newton shifts), each step from basis X_0..X_m (m = columns done):
//   Y_0 = V_m, Y_t = M^{-1}A Y_{t-1} - theta_t Y_{t-1}       (S operator applications)
//   D = X^H Y, C = Rf^{-H} D (projection in V coordinates)   (one sweep of the basis)
//   Y' = Y - X Rf^{-1} C, G = Y'^H Y'                        (one sweep of the basis)
//   G = Rb^H Rb (Cholesky); raw storage: X_{m+1..m+S} = Y', Rf block = Rb;
//   orthonormalised storage: X_{m+1..m+S} = Y' Rb^{-1}, Rf block = I
//   next shifts: Ritz values of this block's S x S diagonal Hessenberg block
// and the Hessenberg columns m..m+S-1 follow from the relations
//   (M^{-1}A) V W_{0:S-1} = V (W_{1:S} + W_{0:S-1} diag(theta)),
// where W holds the V coordinates of Y_0..Y_S (block CA-GMRES change of
// basis).  Givens rotations and the stopping test then run column by column,
// as in gmres() above, so the iteration at which a RHS stops and the iterate
// it returns are those of full GMRES (in exact arithmetic).
// ---------------------------------------------------------------------------
namespace {

// eigenvalues of an n x n complex upper Hessenberg matrix (column-major), shifted QR with deflation
bool hess_eigs(int n, std::vector<cd> A, std::vector<cd>& ev) {
  ev.clear();
  auto a = [&](int i, int j) -> cd& { return A[i + (size_t)j * n]; };
  int hi = n - 1, iter = 0;
  while (hi >= 0) {
    if (hi == 0) {
      ev.push_back(a(0, 0));
      break;
    }
    int l = hi;
    while (l > 0 && std::abs(a(l, l - 1)) > 1e-15 * (std::abs(a(l, l)) + std::abs(a(l - 1, l - 1)))) --l;
    if (l == hi) {
      ev.push_back(a(hi, hi));
      --hi;
      iter = 0;
      continue;
    }
    if (++iter > 100 * n) return false;
    // Wilkinson shift from the trailing 2x2 block of the window [l, hi]
    const cd p = a(hi - 1, hi - 1), q = a(hi - 1, hi), r = a(hi, hi - 1), t = a(hi, hi);
    const cd tr = p + t, det = p * t - q * r, disc = std::sqrt(tr * tr / 4.0 - det);
    const cd m1 = tr / 2.0 + disc, m2 = tr / 2.0 - disc;
    cd mu = std::abs(m1 - t) < std::abs(m2 - t) ? m1 : m2;
    if (iter % 11 == 10) mu += std::abs(a(hi, hi - 1));  // exceptional shift
    std::vector<double> cs(hi - l);
    std::vector<cd> sn(hi - l);
    for (int k = l; k <= hi; ++k) a(k, k) -= mu;
    for (int k = l; k < hi; ++k) {  // A - mu I = Q R, Givens G_k zeroes a(k+1, k)
      const cd x = a(k, k), y = a(k + 1, k);
      const double nr = std::sqrt(std::norm(x) + std::norm(y));
      double c = 1.0;
      cd sg = 0.0;
      if (nr > 0) {
        c = std::abs(x) / nr;
        sg = (std::abs(x) > 0 ? x / std::abs(x) : cd(1.0, 0.0)) * std::conj(y) / nr;
      }
      for (int j = k; j <= hi; ++j) {
        const cd t1 = a(k, j), t2 = a(k + 1, j);
        a(k, j) = c * t1 + sg * t2;
        a(k + 1, j) = -std::conj(sg) * t1 + c * t2;
      }
      cs[k - l] = c;
      sn[k - l] = sg;
    }
    for (int k = l; k < hi; ++k) {  // R Q = R G_l^H ... G_{hi-1}^H
      const double c = cs[k - l];
      const cd sg = sn[k - l];
      for (int i = l; i <= k + 1; ++i) {
        const cd t1 = a(i, k), t2 = a(i, k + 1);
        a(i, k) = c * t1 + std::conj(sg) * t2;
        a(i, k + 1) = -sg * t1 + c * t2;
      }
    }
    for (int k = l; k <= hi; ++k) a(k, k) += mu;
  }
  return true;
}

// Leja ordering: start from the largest modulus, then maximise the product of distances
void leja_order(std::vector<cd>& z) {
  std::vector<cd> out;
  std::vector<bool> used(z.size(), false);
  for (size_t n = 0; n < z.size(); ++n) {
    int best = -1;
    double bv = -1.0;
    for (size_t i = 0; i < z.size(); ++i) {
      if (used[i]) continue;
      double v = 1.0;
      if (out.empty()) v = std::abs(z[i]);
      else
        for (const cd& o : out) v *= std::abs(z[i] - o);
      if (v > bv) {
        bv = v;
        best = (int)i;
      }
    }
    used[best] = true;
    out.push_back(z[best]);
  }
  z = out;
}

// G = R^H R for an n x n Hermitian positive definite G (column-major); false when not positive definite
bool chol_upper(int n, const std::vector<cd>& G, std::vector<cd>& R) {
  R.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    cd d = G[j + (size_t)j * n];
    for (int k = 0; k < j; ++k) d -= std::conj(R[k + (size_t)j * n]) * R[k + (size_t)j * n];
    if (!(d.real() > 0.0) || !std::isfinite(d.real())) return false;
    const double rd = std::sqrt(d.real());
    R[j + (size_t)j * n] = rd;
    for (int i = j + 1; i < n; ++i) {
      cd v = G[j + (size_t)i * n];
      for (int k = 0; k < j; ++k) v -= std::conj(R[k + (size_t)j * n]) * R[k + (size_t)i * n];
      R[j + (size_t)i * n] = v / rd;
    }
  }
  return true;
}

struct BlkState {
  bool active = true, solved = false;
  double beta = 0, eps = 0, rnorm = 0;
  int iters = 0;            // Krylov iterations (Hessenberg columns) taken
  int nvec = 0;             // stored basis vectors
  int ld = 0;               // leading dimension of H and Rf
  std::vector<cd> H;        // V-coordinate Hessenberg, H[i + j*ld]
  std::vector<cd> Rf;       // X = V Rf, Rf[i + k*ld]
  std::vector<int> b0;      // first index of the diagonal block of Rf that holds column k
  std::vector<double> c;    // Givens
  std::vector<cd> s, z;
  std::vector<std::vector<cd>> Rg;
  std::vector<cd> theta;    // Newton shifts
};

// d = Rf^{-1} c over the first K indices (K ends on a block boundary)
void rf_solve(const BlkState& st, int K, const cd* c, cd* d) {
  for (int k = K - 1; k >= 0;) {
    const int a0 = st.b0[k];
    for (int i = k; i >= a0; --i) {
      cd v = c[i];
      for (int j = i + 1; j <= k; ++j) v -= st.Rf[i + (size_t)j * st.ld] * d[j];
      d[i] = v / st.Rf[i + (size_t)i * st.ld];
    }
    k = a0 - 1;
  }
}

// d = Rf^{-H} c over the first K indices
void rf_solve_h(const BlkState& st, int K, const cd* c, cd* d) {
  for (int k0 = 0; k0 < K;) {
    int k1 = k0;
    while (k1 + 1 < K && st.b0[k1 + 1] == k0) ++k1;
    for (int i = k0; i <= k1; ++i) {
      cd v = c[i];
      for (int j = k0; j < i; ++j) v -= std::conj(st.Rf[j + (size_t)i * st.ld]) * d[j];
      d[i] = v / std::conj(st.Rf[i + (size_t)i * st.ld]);
    }
    k0 = k1 + 1;
  }
}

}  // namespace

static int block_size_of(const fm_solve_opts& o) { return o.block > 0 ? o.block : 4; }

template <typename R, typename YR, int S>
static cudaError_t launch_blockdot(fm_plan* P, int nb, int K, const void* U, const void* Y, const int* act, int nact) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  const double bytes = ((double)K * sizeof(T) + (double)S * sizeof(TY)) * nact * P->M;
  const size_t pb =
      P->bd_bulk ? blockdot_bulk_part_bytes((int)sizeof(R), (int)sizeof(YR), S, P->M, nb, nact, K, P->sms) : 0;
  if (pb) {
    cudaError_t e = P->red_part.ensure(pb);
    if (e == cudaSuccess) e = P->red_out.ensure((size_t)nb * (std::max)(K * S, KV_KMAX + 2) * sizeof(double2));
    if (e != cudaSuccess) return e;
    FM_TRACK(P, KC_DOT, bytes,
             e = launch_blockdot_bulk((int)sizeof(R), (int)sizeof(YR), S, P->M, nb, nact, K, U, Y,
                                      (double2*)P->red_part.p, P->red_part.cap, (double2*)P->red_out.p,
                                      (unsigned*)P->red_cnt.p, act, (int*)P->errbuf.p, P->sms, P->st));
    return e;
  }
  auto kern = k_blockdot_mma<R, TY, S>;
  // CTA shape: KW warps along the basis times EW along the elements, with KW * EW <= KV_WARPS and no idle warp
  // (a basis of 9..16 groups of 8 vectors would otherwise leave up to 3 of 8 warps without work)
  const int KG = (K + 7) / 8, GPW = S <= 4 ? 4 : 2, KW = (KG + GPW - 1) / GPW;
  const int threads = 32 * KW * std::max(1, KV_WARPS / KW);
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, threads, 0) != cudaSuccess || bps < 1) bps = 1;
  const long long maxb = (P->M + 127) / 128;
  const int nblk = (int)std::max(1LL, std::min<long long>(maxb, (long long)P->sms * bps / nb));
  cudaError_t e = P->red_part.ensure((size_t)nb * nblk * K * S * sizeof(double2));
  if (e == cudaSuccess) e = P->red_out.ensure((size_t)nb * (std::max)(K * S, KV_KMAX + 2) * sizeof(double2));
  if (e != cudaSuccess) return e;
  FM_TRACK(P, KC_DOT, bytes,
           (kern<<<dim3(nblk, nb), threads, 0, P->st>>>(P->M, nb, K, (const T*)U, (const TY*)Y,
                                                         (double2*)P->red_part.p, (double2*)P->red_out.p,
                                                         (unsigned*)P->red_cnt.p, act)));
  return cudaGetLastError();
}

// Z = Y - X E and the Gram matrix of Z.  TZ: type of Z (the basis type, or the block-vector type when the block
// is stored orthonormalised afterwards and Z overwrites Y in place).  The Gram goes to red_out: the upper triangle
// tri(t,u) for S <= 8 (k_blockgram), the full S x S matrix <Z_t, Z_u> at t*S + u for S > 8 (the block dot of Z
// against itself on the tensor cores).
template <typename R, typename YR, int S, typename TZ>
static cudaError_t launch_blockupdate(fm_plan* P, int nb, int K, const void* U, const void* Y, void* Z, const int* act,
                                      int nact) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  constexpr int NG = S * (S + 1) / 2;
  constexpr int TILE = S <= 8 ? 32 : 16;  // elements per warp tile of k_blockupdate_mma
  constexpr size_t ring = blockupdate_ring_bytes<R, S>();
  auto kern = k_blockupdate_mma<R, TY, S, TZ>;
  // the ring and the static coefficient tile together exceed the default 48 KB a block: opt in
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ring);
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, KV_THREADS, ring) != cudaSuccess || bps < 1) bps = 1;
  const long long maxb = (P->M + TILE * KV_WARPS - 1) / (TILE * KV_WARPS);
  const int nblk = (int)std::max(1LL, std::min<long long>(maxb, (long long)P->sms * bps / nb));
  FM_TRACK(P, KC_UPD, ((double)K * sizeof(T) + (double)S * (sizeof(TY) + sizeof(TZ))) * nact * P->M,
           (kern<<<dim3(nblk, nb), KV_THREADS, ring, P->st>>>(P->M, nb, K, (const T*)U, (const TY*)Y, (TZ*)Z,
                                                               (const double2*)P->coef.p, act)));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if constexpr (S > 8) {
    using ZR = typename RealOf<TZ>::R;
    auto kern = k_blockdot_mma<ZR, TZ, S>;
    const int threads = 32 * KV_WARPS;  // K = S: two groups of 8, one warp along the basis, 8 along the elements
    int bg = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bg, kern, threads, 0) != cudaSuccess || bg < 1) bg = 1;
    const int nblk_g = (int)std::max(1LL, std::min<long long>((P->M + 127) / 128, (long long)P->sms * bg / nb));
    e = P->red_part.ensure((size_t)nb * nblk_g * S * S * sizeof(double2));
    if (e == cudaSuccess) e = P->red_out.ensure((size_t)nb * (std::max)(S * S, KV_KMAX + 2) * sizeof(double2));
    if (e != cudaSuccess) return e;
    FM_TRACK(P, KC_MGS, (double)S * sizeof(TZ) * nact * P->M,
             (kern<<<dim3(nblk_g, nb), threads, 0, P->st>>>(P->M, nb, S, (const cplx<ZR>*)Z, (const TZ*)Z,
                                                             (double2*)P->red_part.p, (double2*)P->red_out.p,
                                                             (unsigned*)P->red_cnt.p, act)));
    return cudaGetLastError();
  } else {
    const int nblk_g = kv_blocks(P, k_blockgram<R, S, TZ>, nb);
    e = P->red_part.ensure((size_t)nb * nblk_g * (std::max)(NG, KV_KMAX + 2) * sizeof(double2));
    if (e != cudaSuccess) return e;
    FM_TRACK(P, KC_MGS, (double)S * sizeof(TZ) * nact * P->M,
             (k_blockgram<R, S, TZ><<<dim3(nblk_g, nb), KV_THREADS, 0, P->st>>>(
                 P->M, nb, (const TZ*)Z, (double2*)P->red_part.p, (double2*)P->red_out.p, (unsigned*)P->red_cnt.p,
                 act)));
    return cudaGetLastError();
  }
}

// V (basis slots) = Z Rb^{-1} for the orthonormalised block storage; coefficients in P->coef
template <typename R, typename YR, int S>
static cudaError_t launch_blocknorm(fm_plan* P, int nb, const void* Z, void* V, const int* act, int nact) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  FM_TRACK(P, KC_AXPBY, (double)S * (sizeof(TY) + sizeof(T)) * nact * P->M,
           (k_blocknorm<R, TY, S><<<dim3(kv_blocks(P, k_blocknorm<R, TY, S>, nb), nb), KV_THREADS, 0, P->st>>>(
               P->M, nb, (const TY*)Z, (const double2*)P->coef.p, (T*)V, act)));
  return cudaGetLastError();
}

// which: 0 block dot, 1 block update into the basis, 2 block update in place into Y, 3 orthonormalisation
template <typename R, typename YR>
static cudaError_t block_kernels(fm_plan* P, int which, int S, int nb, int K, const void* U, const void* Y, void* Z,
                                 const int* act, int nact) {
  using T = cplx<R>;
  using TY = cplx<YR>;
#define FM_BLK(SS)                                                                                     \
  case SS:                                                                                             \
    return which == 0   ? launch_blockdot<R, YR, SS>(P, nb, K, U, Y, act, nact)                        \
           : which == 1 ? launch_blockupdate<R, YR, SS, T>(P, nb, K, U, Y, Z, act, nact)              \
           : which == 2 ? launch_blockupdate<R, YR, SS, TY>(P, nb, K, U, Y, Z, act, nact)             \
                        : launch_blocknorm<R, YR, SS>(P, nb, Y, Z, act, nact);
  switch (S) {
    FM_BLK(2) FM_BLK(3) FM_BLK(4) FM_BLK(5) FM_BLK(6) FM_BLK(7) FM_BLK(8) FM_BLK(16)
    default: return cudaErrorInvalidValue;
  }
#undef FM_BLK
}

// Block vectors are generated and kept in FP64 (YR = double) on FP64 and FP32-storage/FP64-arithmetic plans
// unless the caller asks for the plan's storage type (FM_BLOCK_STORAGE): rounding the raw Krylov vectors to FP32
// before they are orthogonalised is what costs accuracy in an s-step basis.  The orthogonalised block is stored
// in the basis type.
template <typename R, typename YR>
static fm_status gmres_block(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info,
                             double deadline) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  const int S = block_size_of(o);
  const bool ortho_store = o.block_store == FM_BLOCK_FP64_ORTHO;
  const size_t fe = (size_t)P->M;
  const size_t fbytes = (size_t)nb * fe * sizeof(T);
  const int itmax = std::max(1, o.maxiters);
  const int cap = itmax + S + 1;  // stored vectors at most
  if (cap > KV_KMAX) return fail(FM_ERR_UNSUPPORTED, "Krylov basis larger than 128 vectors");
  if ((fe & 3) != 0) return fail(FM_ERR_UNSUPPORTED, "block Gram-Schmidt needs 3*N to be a multiple of 4");
  FM_CK(P->basis.ensure((size_t)cap * fbytes));
  FM_CK(P->scale.ensure((size_t)(KV_KMAX + 1) * nb * sizeof(double)));
  FM_CK(P->active.ensure((size_t)nb * sizeof(int)));
  FM_CK(P->coef.ensure((size_t)nb * KV_KMAX * (std::max)(S, 8) * sizeof(double2)));
  FM_CK(P->shifts.ensure((size_t)nb * sizeof(double2)));
  FM_CK(P->yblk.ensure((size_t)(S + 1) * nb * fe * sizeof(TY)));
  FM_TRY(ensure_reduce(P, nb, KV_KMAX));
  T* U = (T*)P->basis.p;
  TY* Yb = (TY*)P->yblk.p;
  // operator on the block vectors: FP64 potential when the block type is wider than the plan's storage
  RhsCtx rcY;
  rcY.V = P->V.p;
  if (sizeof(TY) != sizeof(T)) {
    FM_CK(P->V64.ensure((size_t)P->n * sizeof(double2)));
    k_to_f64<R><<<2 * P->sms, 256, 0, P->st>>>(P->n, (const T*)P->V.p, 1.0, (double2*)P->V64.p);
    FM_CK(cudaGetLastError());
    rcY.V = P->V64.p;
  }
  double* sc = (double*)P->scale.p;
  int* act = (int*)P->active.p;
  const double btol = std::pow(2.220446049250313e-16, 0.75);
  const int ld = cap + 1;

  std::vector<BlkState> St(nb);
  std::vector<int> acth(nb, 1);
  EpiParams ep{};
  ep.inv_eps = P->kref2 / P->eps_imag;
  auto upload_active = [&]() -> fm_status {
    FM_CK(cudaMemcpyAsync(act, acth.data(), nb * sizeof(int), cudaMemcpyHostToDevice, P->st));
    return FM_OK;
  };
  auto count_active = [&]() {
    int n = 0;
    for (int b = 0; b < nb; ++b) n += acth[b];
    return n;
  };
  // Givens update with Hessenberg column j of RHS r; true when the RHS stops at this column
  auto givens_col = [&](BlkState& r, int j) -> bool {
    const int K = j + 1;
    std::vector<cd> col(K);
    for (int i = 0; i < K; ++i) col[i] = r.H[i + (size_t)j * ld];
    const double hb = r.H[(j + 1) + (size_t)j * ld].real();
    for (int i = 0; i < K - 1; ++i) {
      cd t = r.c[i] * col[i] + r.s[i] * col[i + 1];
      col[i + 1] = std::conj(r.s[i]) * col[i] - r.c[i] * col[i + 1];
      col[i] = t;
    }
    double c;
    cd sn, rho;
    sym_givens(col[K - 1], hb, c, sn, rho);
    col[K - 1] = rho;
    r.c.push_back(c);
    r.s.push_back(sn);
    r.Rg.push_back(col);
    const cd zk1 = std::conj(sn) * r.z[K - 1];
    r.z[K - 1] = c * r.z[K - 1];
    r.rnorm = std::abs(zk1);
    r.iters = K;
    r.solved = (r.rnorm <= r.eps) || (r.rnorm + 1.0 <= 1.0);
    if (r.solved || hb <= btol || K >= itmax) return true;
    r.z.push_back(zk1);
    return false;
  };

  // r0 = M^{-1}(b - A x) into X_0
  FM_TRY(upload_active());
  FM_TRY(green_op<R>(P, nb, P->xbuf.p, PRO_V, nullptr, EPI_PREC_RES, P->xbuf.p, P->bbuf.p, ep, U, act));
  std::vector<double2> hv;
  FM_TRY(multidot<R>(P, nb, 0, U, U, true, act, hv));
  for (int b = 0; b < nb; ++b) {
    BlkState& r = St[b];
    r.ld = ld;
    r.H.assign((size_t)ld * ld, 0.0);
    r.Rf.assign((size_t)ld * ld, 0.0);
    r.b0.assign(ld, 0);
    r.beta = std::sqrt(hv[b].x);
    r.rnorm = r.beta;
    r.eps = o.abstol + o.reltol * r.beta;
    info[b].residual0 = r.beta;
    r.Rf[0] = r.beta;
    r.b0[0] = 0;
    r.nvec = 1;
    r.z.assign(1, cd(r.beta, 0.0));
    if (r.beta == 0.0 || r.rnorm <= r.eps) {
      r.active = false;
      r.solved = true;
      acth[b] = 0;
    }
  }

  // ---- phase 1: S classical Gram-Schmidt steps (Ritz values for the shifts) ----
  int m = 0;  // columns done by the RHS still running
  std::vector<double> sch(nb, 0.0);
  while (count_active() > 0 && m < S && m < itmax) {
    const int nact = count_active();
    FM_TRY(upload_active());
    for (int b = 0; b < nb; ++b) sch[b] = acth[b] ? 1.0 / St[b].Rf[m + (size_t)m * ld].real() : 0.0;
    FM_CK(cudaMemcpyAsync(sc, sch.data(), nb * sizeof(double), cudaMemcpyHostToDevice, P->st));
    T* Uj = U + (size_t)m * nb * fe;
    T* Uw = U + (size_t)(m + 1) * nb * fe;
    FM_TRY(green_op<R>(P, nb, Uj, PRO_V_SCALE, sc, EPI_PREC_OP, Uj, nullptr, ep, Uw, act, nact));
    const int K = m + 1;
    std::vector<double2> hr;
    FM_TRY(multidot<R>(P, nb, K, U, Uw, false, act, hr, nact));
    std::vector<double2> cf((size_t)nb * K, make_double2(0, 0));
    for (int b = 0; b < nb; ++b) {
      if (!acth[b]) continue;
      for (int k = 0; k < K; ++k) {
        const double rk = St[b].Rf[k + (size_t)k * ld].real();
        const cd h = cd(hr[(size_t)b * K + k].x, hr[(size_t)b * K + k].y) / rk;
        St[b].H[k + (size_t)m * ld] = h;
        const cd e = h / rk;
        cf[(size_t)b * K + k] = make_double2(e.real(), e.imag());
      }
    }
    FM_CK(cudaMemcpyAsync(P->coef.p, cf.data(), cf.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
    Coef c{(const double2*)P->coef.p, K, nullptr, nb, -1.0, 0};
    dim3 g(kv_blocks(P, k_update<R, true>, nb), nb);
    FM_TRACK(P, KC_UPD, (double)(K + 2) * nact * fe * sizeof(T),
             (k_update<R, true><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, K, U, c, Uw, nullptr, (double2*)P->red_part.p,
                                                             (double2*)P->red_out.p, (unsigned*)P->red_cnt.p, act)));
    FM_CK(cudaGetLastError());
    std::vector<double2> nn(nb);
    FM_CK(cudaMemcpyAsync(nn.data(), P->red_out.p, nb * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
    tk_resolve(P);
    for (int b = 0; b < nb; ++b) {
      if (!acth[b]) continue;
      BlkState& r = St[b];
      const double hb = std::sqrt(std::max(0.0, nn[b].x));
      r.H[(m + 1) + (size_t)m * ld] = hb;
      r.Rf[(m + 1) + (size_t)(m + 1) * ld] = hb;
      r.b0[m + 1] = m + 1;
      r.nvec = m + 2;
      if (givens_col(r, m)) {
        r.active = false;
        acth[b] = 0;
      }
    }
    ++m;
    if (deadline > 0 && now_s() > deadline) return fail(FM_ERR_TIMEOUT, "solve deadline passed");
  }
  // Newton shifts: Ritz values of the leading S x S Hessenberg block, Leja ordered
  for (int b = 0; b < nb; ++b) {
    BlkState& r = St[b];
    r.theta.assign(S, 0.0);
    if (!r.active) continue;
    std::vector<cd> Hs((size_t)S * S), ev;
    for (int j = 0; j < S; ++j)
      for (int i = 0; i < S; ++i) Hs[i + (size_t)j * S] = r.H[i + (size_t)j * ld];
    if (hess_eigs(S, Hs, ev) && (int)ev.size() == S) {
      leja_order(ev);
      r.theta = ev;
    }
  }

  // ---- phase 2: s-step blocks ----
  while (count_active() > 0 && m < itmax) {
    const int nact = count_active();
    FM_TRY(upload_active());
    const int K = m + 1;
    // Y_0 = V_m = sum_k X_k (Rf^{-1})_{k,m} over m's diagonal block (the same block layout for every RHS)
    int k0 = m;
    for (int b = 0; b < nb; ++b)
      if (acth[b]) k0 = St[b].b0[m];
    const int nc = m - k0 + 1;
    {
      std::vector<double2> cc((size_t)nb * 16, make_double2(0, 0));
      for (int b = 0; b < nb; ++b) {
        if (!acth[b]) continue;
        std::vector<cd> em(K, 0.0), d(K, 0.0);
        em[m] = 1.0;
        rf_solve(St[b], K, em.data(), d.data());
        for (int a2 = 0; a2 < nc; ++a2) cc[(size_t)b * 16 + a2] = make_double2(d[k0 + a2].real(), d[k0 + a2].imag());
      }
      FM_CK(cudaMemcpyAsync(P->coef.p, cc.data(), cc.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_TRACK(P, KC_AXPBY, (double)nc * nact * fe * sizeof(T) + (double)nact * fe * sizeof(TY),
               (k_combine<R, TY><<<dim3(2 * P->sms, nb), KV_THREADS, 0, P->st>>>(
                   P->M, nb, k0, nc, U, (const double2*)P->coef.p, 16, Yb, act)));
      FM_CK(cudaGetLastError());
    }
    // Y_t = M^{-1}A Y_{t-1} - theta_t Y_{t-1}, t = 1..S
    std::vector<double2> th(nb);
    for (int t = 1; t <= S; ++t) {
      for (int b = 0; b < nb; ++b) th[b] = make_double2(St[b].theta[t - 1].real(), St[b].theta[t - 1].imag());
      FM_CK(cudaMemcpyAsync(P->shifts.p, th.data(), nb * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      EpiParams eps = ep;
      eps.shift_b = (const double2*)P->shifts.p;
      TY* Yin = Yb + (size_t)(t - 1) * nb * fe;
      TY* Yout = Yb + (size_t)t * nb * fe;
      // (the shift array is rewritten for the next vector in stream order, after this pass has read it)
      FM_TRY(green_op<YR>(P, nb, Yin, PRO_V, nullptr, EPI_PREC_OP, Yin, nullptr, eps, Yout, act, nact, &rcY));
    }
    // D = X^H Y_{1..S}
    FM_CK((block_kernels<R, YR>(P, 0, S, nb, K, U, Yb + (size_t)nb * fe, nullptr, act, nact)));
    std::vector<double2> D((size_t)nb * K * S);
    FM_CK(cudaMemcpyAsync(D.data(), P->red_out.p, D.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
    tk_resolve(P);
    // C = Rf^{-H} D (V coordinates), E = Rf^{-1} C (X coordinates) for the update
    std::vector<std::vector<cd>> Cv(nb);
    std::vector<double2> cf((size_t)nb * KV_KMAX * S, make_double2(0, 0));
    for (int b = 0; b < nb; ++b) {
      if (!acth[b]) continue;
      Cv[b].assign((size_t)K * S, 0.0);
      std::vector<cd> dcol(K), ccol(K), ecol(K);
      for (int t = 0; t < S; ++t) {
        for (int k = 0; k < K; ++k) {
          const double2 v = D[((size_t)b * K + k) * S + t];
          dcol[k] = cd(v.x, v.y);
        }
        rf_solve_h(St[b], K, dcol.data(), ccol.data());
        rf_solve(St[b], K, ccol.data(), ecol.data());
        for (int k = 0; k < K; ++k) {
          Cv[b][k + (size_t)t * K] = ccol[k];
          cf[(size_t)b * KV_KMAX * S + (size_t)k * S + t] = make_double2(ecol[k].real(), ecol[k].imag());
        }
      }
    }
    FM_CK(cudaMemcpyAsync(P->coef.p, cf.data(), cf.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
    // Y' = Y - X E into basis slots m+1..m+S (orthonormalised storage: over Y in place), Gram of Y'
    if (ortho_store)
      FM_CK((block_kernels<R, YR>(P, 2, S, nb, K, U, Yb + (size_t)nb * fe, Yb + (size_t)nb * fe, act, nact)));
    else
      FM_CK((block_kernels<R, YR>(P, 1, S, nb, K, U, Yb + (size_t)nb * fe, U + (size_t)K * nb * fe, act, nact)));
    // Gram of Y': the upper triangle tri(t,u) per RHS (S <= 8), or the full matrix at t*S + u (S > 8)
    const int NG = S <= 8 ? S * (S + 1) / 2 : S * S;
    std::vector<double2> Gt((size_t)nb * NG);
    FM_CK(cudaMemcpyAsync(Gt.data(), P->red_out.p, Gt.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
    tk_resolve(P);
    std::vector<double2> rbi(ortho_store ? (size_t)nb * S * S : 0, make_double2(0, 0));
    for (int b = 0; b < nb; ++b) {
      if (!acth[b]) continue;
      BlkState& r = St[b];
      std::vector<cd> G((size_t)S * S), Rb;
      int gi = 0;
      for (int t = 0; t < S; ++t)
        for (int u = t; u < S; ++u, ++gi) {
          const size_t at = (size_t)b * NG + (S <= 8 ? (size_t)gi : (size_t)t * S + u);
          const cd v(Gt[at].x, Gt[at].y);
          G[t + (size_t)u * S] = v;
          G[u + (size_t)t * S] = std::conj(v);
        }
      if (!chol_upper(S, G, Rb)) {  // the block lost rank: Krylov breakdown, keep the columns so far
        r.active = false;
        acth[b] = 0;
        continue;
      }
      if (ortho_store) {
        // stored columns V = Y' Rb^{-1} are orthonormal: identity diagonal blocks of Rf
        for (int t = 0; t < S; ++t) {
          std::vector<cd> col(S, 0.0);
          col[t] = 1.0;
          for (int i = t; i >= 0; --i) {
            cd v = col[i];
            for (int q = i + 1; q <= t; ++q) v -= Rb[i + (size_t)q * S] * col[q];
            col[i] = v / Rb[i + (size_t)i * S];
          }
          for (int u = 0; u <= t; ++u) rbi[(size_t)b * S * S + u * S + t] = make_double2(col[u].real(), col[u].imag());
        }
        for (int u = 0; u < S; ++u) {
          for (int a = 0; a <= u; ++a) r.Rf[(K + a) + (size_t)(K + u) * ld] = (a == u) ? cd(1.0, 0.0) : cd(0.0, 0.0);
          r.b0[K + u] = K + u;
        }
      } else {
        for (int u = 0; u < S; ++u) {
          for (int a = 0; a <= u; ++a) r.Rf[(K + a) + (size_t)(K + u) * ld] = Rb[a + (size_t)u * S];
          r.b0[K + u] = K;
        }
      }
      r.nvec = K + S;
      // W: V coordinates of Y_0..Y_S, n x (S+1)
      const int n = K + S;
      std::vector<cd> W((size_t)n * (S + 1), 0.0);
      W[m] = 1.0;  // Y_0 = V_m
      for (int t = 0; t < S; ++t) {
        for (int i = 0; i < K; ++i) W[i + (size_t)(t + 1) * n] = Cv[b][i + (size_t)t * K];
        for (int a = 0; a < S; ++a) W[K + a + (size_t)(t + 1) * n] = Rb[a + (size_t)t * S];
      }
      // Rh = W[:,1:S] + W[:,0:S-1] diag(theta) - [H_{0:m,0:m-1} W_{0:m-1,0:S-1}; 0]
      std::vector<cd> Rh((size_t)n * S), Hn((size_t)n * S);
      for (int c = 0; c < S; ++c) {
        for (int i = 0; i < n; ++i) Rh[i + (size_t)c * n] = W[i + (size_t)(c + 1) * n] + r.theta[c] * W[i + (size_t)c * n];
        for (int j = 0; j < m; ++j) {
          const cd w = W[j + (size_t)c * n];
          if (w == cd(0.0, 0.0)) continue;
          for (int i = 0; i <= j + 1; ++i) Rh[i + (size_t)c * n] -= r.H[i + (size_t)j * ld] * w;
        }
      }
      // Hn = Rh T^{-1}, T = W[m..m+S-1, 0..S-1] upper triangular
      for (int c = 0; c < S; ++c)
        for (int i = 0; i < n; ++i) {
          cd v = Rh[i + (size_t)c * n];
          for (int a = 0; a < c; ++a) v -= Hn[i + (size_t)a * n] * W[m + a + (size_t)c * n];
          Hn[i + (size_t)c * n] = v / W[m + c + (size_t)c * n];
        }
      for (int c = 0; c < S; ++c)
        for (int i = 0; i < n; ++i) r.H[i + (size_t)(m + c) * ld] = (i <= m + c + 1) ? Hn[i + (size_t)c * n] : cd(0.0, 0.0);
      // Newton shifts of the next block: Ritz values of this block's S x S diagonal Hessenberg block, Leja ordered.
      // Shifts kept from the first S steps only let the basis of a later block lose conditioning; refreshed ones
      // keep it near that of s = 4 up to s = 16 (a numpy restatement with FP32-rounded basis vectors on the CBS
      // operator: 4.6e-6 -> 6e-8 at s = 8).
      {
        std::vector<cd> Hs((size_t)S * S), ev;
        for (int j = 0; j < S; ++j)
          for (int i = 0; i < S; ++i) Hs[i + (size_t)j * S] = r.H[(m + i) + (size_t)(m + j) * ld];
        if (hess_eigs(S, Hs, ev) && (int)ev.size() == S) {
          leja_order(ev);
          r.theta = ev;
        }
      }
      for (int c = 0; c < S; ++c) {
        if (givens_col(r, m + c)) {
          r.active = false;
          acth[b] = 0;
          break;
        }
      }
    }
    if (ortho_store) {  // zero coefficients for right-hand sides whose block broke down: their slots stay unused
      FM_CK(cudaMemcpyAsync(P->coef.p, rbi.data(), rbi.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_CK((block_kernels<R, YR>(P, 3, S, nb, K, U, Yb + (size_t)nb * fe, U + (size_t)K * nb * fe, act, nact)));
    }
    m += S;
    if (deadline > 0 && now_s() > deadline) return fail(FM_ERR_TIMEOUT, "solve deadline passed");
  }

  // ---- x += V y = X Rf^{-1} y ----
  std::vector<double2> yh((size_t)nb * KV_KMAX, make_double2(0, 0));
  int Kmax = 0;
  for (int b = 0; b < nb; ++b) {
    BlkState& r = St[b];
    const int n_in = r.iters;
    if (n_in == 0) continue;
    std::vector<cd> y(r.z.begin(), r.z.begin() + n_in);
    for (int i = n_in - 1; i >= 0; --i) {
      for (int jj = n_in - 1; jj > i; --jj) y[i] -= r.Rg[jj][i] * y[jj];
      if (std::abs(r.Rg[i][i]) <= btol) {
        for (int q = 0; q <= i; ++q) y[q] = 0.0;
        break;
      }
      y[i] /= r.Rg[i][i];
    }
    std::vector<cd> yv(r.nvec, 0.0), d(r.nvec, 0.0);
    for (int i = 0; i < n_in; ++i) yv[i] = y[i];
    rf_solve(r, r.nvec, yv.data(), d.data());
    for (int i = 0; i < r.nvec; ++i) yh[(size_t)b * KV_KMAX + i] = make_double2(d[i].real(), d[i].imag());
    Kmax = std::max(Kmax, r.nvec);
  }
  if (Kmax > 0) {
    FM_CK(cudaMemcpyAsync(P->coef.p, yh.data(), yh.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
    Coef cf{(const double2*)P->coef.p, KV_KMAX, nullptr, nb, 1.0, 1};
    dim3 g(kv_blocks(P, k_update<R, false>, nb), nb);
    FM_TRACK(P, KC_UPD, (double)(Kmax + 2) * nb * fe * sizeof(T),
             (k_update<R, false><<<g, KV_THREADS, 0, P->st>>>(P->M, nb, Kmax, U, cf, (T*)P->xbuf.p, nullptr, nullptr,
                                                              nullptr, nullptr, nullptr)));
    FM_CK(cudaGetLastError());
  }
  for (int b = 0; b < nb; ++b) {
    info[b].iterations = St[b].iters;
    info[b].solved = St[b].solved ? 1 : 0;
    info[b].residual = St[b].rnorm;
  }
  return FM_OK;
}

// ---------------------------------------------------------------------------
// BiCGStab (left preconditioned, Krylov.jl form, shadow c = b) and the plain
// Born series (Richardson) on the same operator.
// ---------------------------------------------------------------------------
template <typename R>
static fm_status bicgstab(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info, double deadline) {
  using T = cplx<R>;
  const size_t fe = (size_t)P->M, fbytes = (size_t)nb * fe * sizeof(T);
  // r, p, v, s, t, dx in the basis buffer
  FM_CK(P->basis.ensure(6 * fbytes));
  FM_CK(P->active.ensure((size_t)nb * sizeof(int)));
  T* base = (T*)P->basis.p;
  T *r = base, *p = base + nb * fe, *v = base + 2 * nb * fe, *s = base + 3 * nb * fe, *t = base + 4 * nb * fe,
    *dx = base + 5 * nb * fe;
  int* act = (int*)P->active.p;
  std::vector<int> acth(nb, 1);
  EpiParams ep{};
  ep.inv_eps = P->kref2 / P->eps_imag;
  FM_CK(cudaMemcpyAsync(act, acth.data(), nb * sizeof(int), cudaMemcpyHostToDevice, P->st));
  FM_TRY(green_op<R>(P, nb, P->xbuf.p, PRO_V, nullptr, EPI_PREC_RES, P->xbuf.p, P->bbuf.p, ep, r, act));
  FM_CK(cudaMemcpyAsync(p, r, fbytes, cudaMemcpyDeviceToDevice, P->st));
  FM_CK(cudaMemsetAsync(dx, 0, fbytes, P->st));
  std::vector<double2> hv;
  FM_TRY(multidot<R>(P, nb, 1, P->bbuf.p, r, true, act, hv));  // <c, r>, ||r||^2
  std::vector<cd> rho(nb), next_rho(nb), alpha(nb), omega(nb);
  std::vector<double> rn(nb), eps(nb);
  std::vector<int> iters(nb, 0);
  std::vector<bool> solved(nb, false), active(nb, true);
  for (int b = 0; b < nb; ++b) {
    rn[b] = std::sqrt(hv[2 * b + 1].x);
    info[b].residual0 = rn[b];
    eps[b] = o.abstol + o.reltol * rn[b];
    next_rho[b] = cd(hv[2 * b].x, hv[2 * b].y);
    if (rn[b] == 0.0 || rn[b] <= eps[b]) { solved[b] = true; active[b] = false; }
    else if (next_rho[b] == 0.0) { active[b] = false; }
  }
  auto sync_active = [&]() -> fm_status {
    bool any = false;
    for (int b = 0; b < nb; ++b) { acth[b] = active[b] ? 1 : 0; any |= active[b]; }
    FM_CK(cudaMemcpyAsync(act, acth.data(), nb * sizeof(int), cudaMemcpyHostToDevice, P->st));
    return any ? FM_OK : FM_NOT_CONVERGED;  // NOT_CONVERGED used as "nothing left" sentinel
  };
  int iter = 0;
  std::vector<cd> one(nb, 1.0), z(nb);
  while (iter < o.maxiters) {
    if (sync_active() != FM_OK) break;
    ++iter;
    for (int b = 0; b < nb; ++b) rho[b] = next_rho[b];
    FM_TRY(green_op<R>(P, nb, p, PRO_V, nullptr, EPI_PREC_OP, p, nullptr, ep, v, act));
    FM_TRY(multidot<R>(P, nb, 1, P->bbuf.p, v, false, act, hv));
    std::vector<cd> ma(nb), a(nb);
    for (int b = 0; b < nb; ++b) {
      if (!active[b]) continue;
      alpha[b] = rho[b] / cd(hv[b].x, hv[b].y);
      ma[b] = -alpha[b];
      a[b] = alpha[b];
    }
    FM_TRY(axpby3<R>(P, nb, r, one, v, ma, nullptr, z, s, false, act, nullptr));   // s = r - alpha v
    FM_TRY(axpby3<R>(P, nb, dx, one, p, a, nullptr, z, dx, false, act, nullptr));  // dx += alpha p
    FM_TRY(green_op<R>(P, nb, s, PRO_V, nullptr, EPI_PREC_OP, s, nullptr, ep, t, act));
    std::vector<double2> ts, tt;
    FM_TRY(multidot<R>(P, nb, 1, t, s, false, act, ts));
    FM_TRY(multidot<R>(P, nb, 1, t, t, false, act, tt));
    std::vector<cd> om(nb), mom(nb), beta(nb);
    for (int b = 0; b < nb; ++b) {
      if (!active[b]) continue;
      omega[b] = cd(ts[b].x, ts[b].y) / cd(tt[b].x, tt[b].y);
      om[b] = omega[b];
      mom[b] = -omega[b];
    }
    FM_TRY(axpby3<R>(P, nb, dx, one, s, om, nullptr, z, dx, false, act, nullptr));  // dx += omega s
    std::vector<double> nr;
    FM_TRY(axpby3<R>(P, nb, s, one, t, mom, nullptr, z, r, true, act, &nr));        // r = s - omega t
    FM_TRY(multidot<R>(P, nb, 1, P->bbuf.p, r, false, act, hv));
    for (int b = 0; b < nb; ++b) {
      if (!active[b]) continue;
      next_rho[b] = cd(hv[b].x, hv[b].y);
      beta[b] = (next_rho[b] / rho[b]) * (alpha[b] / omega[b]);
    }
    // p = r + beta (p - omega v)
    std::vector<cd> bm(nb), bw(nb);
    for (int b = 0; b < nb; ++b) { bm[b] = beta[b]; bw[b] = -beta[b] * omega[b]; }
    FM_TRY(axpby3<R>(P, nb, r, one, p, bm, v, bw, p, false, act, nullptr));
    for (int b = 0; b < nb; ++b) {
      if (!active[b]) continue;
      rn[b] = std::sqrt(nr[b]);
      iters[b] = iter;
      const bool ok = rn[b] <= eps[b] || (rn[b] + 1.0 <= 1.0);
      solved[b] = ok;
      if (ok || alpha[b] == 0.0 || std::isnan(alpha[b].real())) active[b] = false;
    }
    if (deadline > 0 && now_s() > deadline) return fail(FM_ERR_TIMEOUT, "solve deadline passed");
  }
  // x = x0 + dx
  std::vector<cd> onev(nb, 1.0);
  FM_TRY(axpby3<R>(P, nb, P->xbuf.p, onev, dx, onev, nullptr, z, P->xbuf.p, false, nullptr, nullptr));
  for (int b = 0; b < nb; ++b) {
    info[b].iterations = iters[b];
    info[b].solved = solved[b] ? 1 : 0;
    info[b].residual = rn[b];
  }
  return FM_OK;
}

template <typename R>
static fm_status richardson(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info,
                            double deadline) {
  using T = cplx<R>;
  const size_t fe = (size_t)P->M, fbytes = (size_t)nb * fe * sizeof(T);
  FM_CK(P->basis.ensure(fbytes));
  FM_CK(P->active.ensure((size_t)nb * sizeof(int)));
  T* r = (T*)P->basis.p;
  int* act = (int*)P->active.p;
  std::vector<int> acth(nb, 1);
  EpiParams ep{};
  ep.inv_eps = P->kref2 / P->eps_imag;
  std::vector<double> rn(nb), eps(nb);
  std::vector<int> iters(nb, 0);
  std::vector<bool> solved(nb, false), active(nb, true);
  std::vector<cd> one(nb, 1.0), z(nb);
  std::vector<double2> hv;
  int iter = 0;
  while (true) {
    bool any = false;
    for (int b = 0; b < nb; ++b) { acth[b] = active[b] ? 1 : 0; any |= active[b]; }
    if (!any) break;
    FM_CK(cudaMemcpyAsync(act, acth.data(), nb * sizeof(int), cudaMemcpyHostToDevice, P->st));
    FM_TRY(green_op<R>(P, nb, P->xbuf.p, PRO_V, nullptr, EPI_PREC_RES, P->xbuf.p, P->bbuf.p, ep, r, act));
    FM_TRY(multidot<R>(P, nb, 0, r, r, true, act, hv));
    for (int b = 0; b < nb; ++b) {
      if (!active[b]) continue;
      rn[b] = std::sqrt(hv[b].x);
      if (iter == 0) { eps[b] = o.abstol + o.reltol * rn[b]; info[b].residual0 = rn[b]; }
      iters[b] = iter;
      if (rn[b] <= eps[b]) { solved[b] = true; active[b] = false; }
      else if (iter >= o.maxiters) active[b] = false;
      acth[b] = active[b] ? 1 : 0;
    }
    FM_CK(cudaMemcpyAsync(act, acth.data(), nb * sizeof(int), cudaMemcpyHostToDevice, P->st));
    FM_TRY(axpby3<R>(P, nb, P->xbuf.p, one, r, one, nullptr, z, P->xbuf.p, false, act, nullptr));
    ++iter;
    if (deadline > 0 && now_s() > deadline) return fail(FM_ERR_TIMEOUT, "solve deadline passed");
  }
  for (int b = 0; b < nb; ++b) {
    info[b].iterations = iters[b];
    info[b].solved = solved[b] ? 1 : 0;
    info[b].residual = rn[b];
  }
  return FM_OK;
}

// reads (and clears) the device error code set by bounded pipeline waits
static fm_status check_device_error(fm_plan* P) {
  int code = 0;
  FM_CK(cudaMemcpyAsync(&code, P->errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  if (code) {
    cudaMemsetAsync(P->errbuf.p, 0, sizeof(int), P->st);
    return fail(FM_ERR_TIMEOUT, "a TMA pipeline wait timed out on the device (code " + std::to_string(code) + ")");
  }
  return FM_OK;
}

// H = -i lambda/(2 pi 377) curl(E) for nb fields (in -> out, both contiguous batches; act masks RHS)
template <typename R>
static fm_status curl_batch(fm_plan* P, int nb, const void* in, void* out, const int* act) {
  using T = cplx<R>;
  const size_t fbytes = (size_t)nb * P->M * sizeof(T);
  EpiParams ep{};
  Dims d = P->dims;
  d.nb = nb;
  FM_CK(P->t1.ensure(fbytes));
  FM_CK(P->t2.ensure(fbytes));
  GreenParams gp{};
  for (int a = 0; a < 3; ++a)
    gp.dk[a] = 2.0 * M_PI / ((double)(a == 0 ? d.nx : a == 1 ? d.ny : d.nz) * P->desc.resolution[a]);
  const double f = P->wavelength / (2.0 * M_PI * 377.0) / (double)P->n;
  gp.scale_re = 0.0;
  gp.scale_im = -f;
  const double cb = 2.0 * nb * P->M * sizeof(T);
  cudaError_t e;
  if (P->generic) {
    GenRamps none;
    FM_TRACK(P, KC_CURL, cb, e = gen_pre<R>(P, d, PRO_COPY, in, nullptr, nullptr, none, P->t1.p, act, VecTab{}));
    FM_CK(e);
    for (int a = 0; a < 3; ++a) {
      FM_TRACK(P, KC_CURL, cb, e = gen_axis<R>(P, d, a, -1, P->t1.p, act));
      FM_CK(e);
    }
    FM_TRACK(P, KC_CURL, cb, e = gen_kspace<R>(P, d, ZMODE_CURL, P->t1.p, gp, act));
    FM_CK(e);
    for (int a = 2; a >= 0; --a) {
      FM_TRACK(P, KC_CURL, cb, e = gen_axis<R>(P, d, a, +1, P->t1.p, act));
      FM_CK(e);
    }
    FM_TRACK(P, KC_CURL, cb,
             e = gen_post<R>(P, d, EPI_STORE, P->t1.p, nullptr, nullptr, nullptr, nullptr, ep, none, out, act, VecTab{}));
    FM_CK(e);
    return FM_OK;
  }
  FM_TRACK(P, KC_CURL, cb, e = pass_xf<R>(P, d, PRO_COPY, in, nullptr, nullptr, P->twx.p, nullptr, P->t1.p, act));
  FM_CK(e);
  FM_TRACK(P, KC_CURL, cb, e = pass_y<R>(P, d, -1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
  FM_CK(e);
  FM_TRACK(P, KC_CURL, cb, e = pass_zg<R>(P, d, ZMODE_CURL, P->t2.p, gp, P->twz.p, nullptr, P->t1.p, act));
  FM_CK(e);
  FM_TRACK(P, KC_CURL, cb, e = pass_y<R>(P, d, +1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
  FM_CK(e);
  FM_TRACK(P, KC_CURL, cb,
           e = pass_xi<R>(P, d, EPI_STORE, P->t2.p, nullptr, nullptr, nullptr, nullptr, ep, P->twx.p, nullptr,
                            out, act));
  FM_CK(e);
  return FM_OK;
}

// ---------------------------------------------------------------------------
// shared solve core: from scaled source terms in P->sbuf (nb RHS) to the
// scattered field in P->xbuf and its curl in P->ebuf.
// ---------------------------------------------------------------------------
template <typename R>
static fm_status solve_core(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info) {
  using T = cplx<R>;
  const size_t fbytes = (size_t)nb * P->M * sizeof(T);
  const double deadline = o.timeout_s > 0 ? now_s() + o.timeout_s : 0.0;
  FM_CK(P->bbuf.ensure(fbytes));
  FM_CK(P->xbuf.ensure(fbytes));
  FM_CK(P->ebuf.ensure(fbytes));
  EpiParams ep{};
  // b = G_avg S ; x0 = b
  FM_TRY(green_op<R>(P, nb, P->sbuf.p, PRO_COPY, nullptr, EPI_STORE, nullptr, nullptr, ep, P->bbuf.p, nullptr));
  FM_CK(cudaMemcpyAsync(P->xbuf.p, P->bbuf.p, fbytes, cudaMemcpyDeviceToDevice, P->st));
  fm_status st;
  if (o.method == FM_METHOD_GMRES && o.ortho == FM_ORTHO_BLOCK)
    st = (P->c64 && o.block_store != FM_BLOCK_STORAGE) ? gmres_block<R, double>(P, nb, o, info, deadline)
                                                    : gmres_block<R, R>(P, nb, o, info, deadline);
  else if (o.method == FM_METHOD_GMRES) st = gmres<R>(P, nb, o, info, deadline);
  else if (o.method == FM_METHOD_BICGSTAB) st = bicgstab<R>(P, nb, o, info, deadline);
  else if (o.method == FM_METHOD_RICHARDSON) st = richardson<R>(P, nb, o, info, deadline);
  else return fail(FM_ERR_INVALID, "unknown method");
  if (st != FM_OK) return st;
  // H_s = -i lambda/(2 pi 377) curl(E_s)
  FM_TRY(curl_batch<R>(P, nb, P->xbuf.p, P->ebuf.p, nullptr));
  return check_device_error(P);
}

// ---------------------------------------------------------------------------
// host <-> device conversions
// ---------------------------------------------------------------------------
template <typename R>
static fm_status h2d_field(fm_plan* P, const double* host, long long count, double s, void* dst) {
  FM_CK(P->gbuf2.ensure((size_t)count * sizeof(double2)));
  FM_CK(cudaMemcpyAsync(P->gbuf2.p, host, (size_t)count * sizeof(double2), cudaMemcpyHostToDevice, P->st));
  k_from_f64<R><<<1184, 256, 0, P->st>>>(count, (const double2*)P->gbuf2.p, s, (cplx<R>*)dst);
  FM_CK(cudaGetLastError());
  return FM_OK;
}
template <typename R>
static fm_status d2h_field(fm_plan* P, const void* src, long long count, double s, double* host) {
  FM_CK(P->gbuf2.ensure((size_t)count * sizeof(double2)));
  k_to_f64<R><<<1184, 256, 0, P->st>>>(count, (const cplx<R>*)src, s, (double2*)P->gbuf2.p);
  FM_CK(cudaGetLastError());
  FM_CK(cudaMemcpyAsync(host, P->gbuf2.p, (size_t)count * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  return FM_OK;
}

static fm_status check_plan(fm_plan* P, int nrhs, bool need_pot) {
  if (!P) return fail(FM_ERR_INVALID, "null plan");
  if (nrhs < 1) return fail(FM_ERR_INVALID, "nrhs must be >= 1");
  if (need_pot && !P->have_pot) return fail(FM_ERR_INVALID, "potential not set (fm_set_potential / fm_build_potential)");
  FM_CK(cudaSetDevice(P->desc.device));
  return FM_OK;
}

static fm_status validate_opts(const fm_solve_opts* o) {
  if (!o) return fail(FM_ERR_INVALID, "null options");
  if (o->maxiters < 1) return fail(FM_ERR_INVALID, "maxiters must be >= 1");
  if (!(o->reltol >= 0 && o->reltol <= 1)) return fail(FM_ERR_INVALID, "tolerance must be in [0, 1]");
  if (!(o->abstol >= 0)) return fail(FM_ERR_INVALID, "abstol must be >= 0");
  if (o->method < 0 || o->method > 2) return fail(FM_ERR_INVALID, "unknown method");
  if (o->ortho < 0 || o->ortho > 3) return fail(FM_ERR_INVALID, "unknown orthogonalisation");
  if (o->ortho == FM_ORTHO_BLOCK && o->method == FM_METHOD_GMRES) {
    if (o->block != 0 && (o->block < 2 || (o->block > 8 && o->block != 16)))
      return fail(FM_ERR_INVALID, "block size must be 2..8 or 16");
    if (o->block_store != FM_BLOCK_FP64 && o->block_store != FM_BLOCK_STORAGE && o->block_store != FM_BLOCK_FP64_ORTHO)
      return fail(FM_ERR_INVALID, "unknown block vector storage");
    if (o->restart > 0) return fail(FM_ERR_UNSUPPORTED, "block GMRES runs full GMRES only (restart = 0)");
    if (o->maxiters + block_size_of(*o) + 1 > KV_KMAX)
      return fail(FM_ERR_UNSUPPORTED, "GMRES basis larger than 128 vectors");
  }
  if (o->restart < 0) return fail(FM_ERR_INVALID, "restart must be >= 0");
  if (o->method == FM_METHOD_GMRES) {
    const int mem = o->restart > 0 ? std::min(o->restart, o->maxiters) : o->maxiters;
    if (mem + 1 > KV_KMAX) return fail(FM_ERR_UNSUPPORTED, "GMRES basis larger than 127 vectors (use restart)");
  }
  return FM_OK;
}

template <typename R>
static fm_status plan_wave_size(fm_plan* P, int nrhs, const fm_solve_opts& o, int& wave) {
  size_t freeb = 0, totalb = 0;
  FM_CK(cudaMemGetInfo(&freeb, &totalb));
  const size_t fb = (size_t)P->M * sizeof(cplx<R>);
  int vecs = 0;
  if (o.method == FM_METHOD_GMRES) vecs = (o.restart > 0 ? std::min(o.restart, o.maxiters) : o.maxiters) + 1;
  size_t extra = 0;  // block GMRES: FP64 block vectors, FP64 pass temporaries, FP64 potential
  if (o.method == FM_METHOD_GMRES && o.ortho == FM_ORTHO_BLOCK) {
    vecs = o.maxiters + block_size_of(o) + 1;
    extra = (o.block_store != FM_BLOCK_STORAGE && P->c64) ? (size_t)P->M * sizeof(double2) * (block_size_of(o) + 1 + 2)
                                                        : fb * (size_t)(block_size_of(o) + 1);
  }
  else if (o.method == FM_METHOD_BICGSTAB) vecs = 6;
  else vecs = 1;
  // basis + b + x + s + e + t1 + t2 + fp64 staging and outputs
  // (the output term also covers the second output slot of host-output solves: 2 * 3g * 16 <= 2 * M * 16)
  // (+ t3 when the Green average runs as two branches: absorbing x or y)
  const size_t two_branch = (P->avg && !P->zonly && !P->zsplit) ? 1 : 0;  // (the general passes use t1 and t3)
  const size_t per = fb * (size_t)(vecs + 6 + two_branch) + (size_t)P->M * sizeof(double2) * 5 + extra;
  const size_t held = P->basis.cap + P->bbuf.cap + P->xbuf.cap + P->sbuf.cap + P->ebuf.cap + P->t1.cap + P->t2.cap +
                      P->t3.cap +
                      P->gbuf2.cap + P->Eo.cap + P->Ho.cap + P->yblk.cap;
  const size_t avail = (size_t)((freeb + held) * 0.92);
  wave = (int)std::max<size_t>(1, std::min<size_t>((size_t)nrhs, avail / per));
  wave = std::min(wave, std::max(1, P->desc.max_rhs));
  if (P->wave_rhs > 0) wave = std::min(wave, P->wave_rhs);
  // balance the waves: ceil(nrhs / waves) right-hand sides each
  const int waves = (nrhs + wave - 1) / wave;
  wave = (nrhs + waves - 1) / waves;
  if ((size_t)wave * per > avail) return fail(FM_ERR_OOM, "one right-hand side does not fit in device memory");
  return FM_OK;
}

// ---------------------------------------------------------------------------
// C ABI (C linkage comes from the declarations in fmcuda.h)
// ---------------------------------------------------------------------------

int fm_abi_version(void) { return FMCUDA_ABI_VERSION; }
const char* fm_last_error(void) { return g_err.c_str(); }
int fm_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

long long fm_plan_bytes(const fm_plan_desc* d, int nrhs, int basis) {
  if (!d) return -1;
  long long n = 1;
  for (int a = 0; a < 3; ++a) n *= (long long)(d->grid[a] + 2 * d->pad[a]);
  const long long fb = 3 * n * (d->precision == FM_PREC_F64 ? 16 : 8);
  // basis + six work fields per right-hand side, the potential, and the FP64 E/H outputs in two slots (host
  // outputs are copied from one slot while the next wave fills the other)
  return fb * (long long)nrhs * (basis + 6) + n * (d->precision == FM_PREC_F64 ? 16 : 8) +
         4LL * 3 * n * 16 * nrhs;
}

fm_status fm_plan_create(const fm_plan_desc* desc, fm_plan** out) {
  if (!desc || !out) return fail(FM_ERR_INVALID, "null argument");
  *out = nullptr;
  for (int a = 0; a < 3; ++a) {
    if (desc->grid[a] <= 0) return fail(FM_ERR_INVALID, "all grid_size components must be positive");
    if (desc->pad[a] < 0) return fail(FM_ERR_INVALID, "padding must be >= 0");
    if (!(desc->resolution[a] > 0)) return fail(FM_ERR_INVALID, "all resolution components must be positive");
  }
  if (desc->precision != FM_PREC_F32 && desc->precision != FM_PREC_F64 && desc->precision != FM_PREC_F32_MATH64)
    return fail(FM_ERR_INVALID, "precision must be FM_PREC_F32, FM_PREC_F64 or FM_PREC_F32_MATH64");
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) return fail(FM_ERR_CUDA, "no CUDA device");
  if (desc->device < 0 || desc->device >= nd) return fail(FM_ERR_INVALID, "device ordinal out of range");
  const int n3[3] = {desc->grid[0] + 2 * desc->pad[0], desc->grid[1] + 2 * desc->pad[1], desc->grid[2] + 2 * desc->pad[2]};
  bool avg = desc->absorbing[0] || desc->absorbing[1] || desc->absorbing[2];
  bool zonly = desc->absorbing[2] && !desc->absorbing[0] && !desc->absorbing[1];
  const int prec = desc->precision == FM_PREC_F64 ? FM_PREC_F64 : FM_PREC_F32;  // storage
  const bool c64 = desc->precision != FM_PREC_F32;                                   // arithmetic
  // The fused passes take axes of 96 or powers of two in [8, 512] (an averaged z axis a power of two) that
  // tile the warps; every other grid runs the general passes (fm_generic.cuh).
  bool generic = false;
  for (int a = 0; a < 3; ++a)
    if (!axis_supported(n3[a])) generic = true;
  if (zonly && (n3[2] > AXIS_MAX || (n3[2] & (n3[2] - 1)))) generic = true;
  // padded z above 256: the two shifted branches run as two z passes (the second adds to the first)
  bool zsplit = zonly && n3[2] > AXIS_MAX_AVG2;
  if (!generic) {
    const int pwy = c64 ? pencils_per_warp<double>(n3[1]) : pencils_per_warp<float>(n3[1]);
    const int lz = (zonly && !zsplit) ? 2 * n3[2] : n3[2];
    const int pwz = c64 ? pencils_per_warp<double>(lz) : pencils_per_warp<float>(lz);
    if (pwy <= 0 || pwz <= 0 || n3[0] % pwy || n3[0] % pwz) generic = true;
  }
  if (generic) {
    for (int a = 0; a < 3; ++a)
      if (!gen_axis_supported(n3[a]))
        return fail(FM_ERR_UNSUPPORTED, "padded axis sizes must be at most 256, or powers of two up to 512");
    zonly = zsplit = false;
  }
  if (cudaSetDevice(desc->device) != cudaSuccess) return fail(FM_ERR_CUDA, "cudaSetDevice failed");
  fm_plan* P = new fm_plan();
  P->desc = *desc;
  if (P->desc.max_rhs < 1) P->desc.max_rhs = 1;
  P->prec = prec;
  P->c64 = c64;
  P->esz = prec == FM_PREC_F64 ? 16 : 8;
  P->dims = Dims{n3[0], n3[1], n3[2], 1, (long long)n3[0] * n3[1] * n3[2]};
  P->n = P->dims.n;
  P->M = 3 * P->n;
  P->pi = PadInfo{desc->grid[0], desc->grid[1], desc->grid[2], desc->pad[0], desc->pad[1], desc->pad[2], n3[0], n3[1], n3[2]};
  P->avg = avg;
  P->zonly = zonly && !zsplit;
  P->zsplit = zsplit;
  P->generic = generic;
  for (int a = 0; a < 3; ++a) P->shift[a] = desc->absorbing[a] ? 0.25 : 0.0;
  {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, desc->device) == cudaSuccess) P->sms = prop.multiProcessorCount;
  }
  if (cudaStreamCreateWithFlags(&P->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete P;
    return fail(FM_ERR_CUDA, "stream creation failed");
  }
  {
    const char* no_tma = std::getenv("FMCUDA_NO_TMA");
    P->use_tma = !(no_tma && no_tma[0] == '1');
  }
  if (P->errbuf.ensure(sizeof(int)) != cudaSuccess || cudaMemsetAsync(P->errbuf.p, 0, sizeof(int), P->st) != cudaSuccess) {
    fm_plan_destroy(P);
    return fail(FM_ERR_CUDA, "error-flag allocation failed");
  }
  fm_status s = c64 ? init_tables<double>(P) : init_tables<float>(P);
  if (s != FM_OK) {
    fm_plan_destroy(P);
    return s;
  }
  *out = P;
  return FM_OK;
}

void fm_plan_destroy(fm_plan* P) {
  if (!P) return;
  cudaSetDevice(P->desc.device);
  if (P->st) cudaStreamSynchronize(P->st);
  DevBuf* bufs[] = {&P->twx, &P->twy, &P->twz, &P->twz2, &P->rz, &P->rxp, &P->rxm, &P->ryp, &P->rym, &P->rzp,
                    &P->rzm, &P->V, &P->t1, &P->t2, &P->t3, &P->bbuf, &P->xbuf, &P->ebuf, &P->sbuf, &P->basis,
                    &P->gbuf2, &P->red_part, &P->red_out, &P->red_cnt, &P->active, &P->scale, &P->coef,
                    &P->hbuf, &P->eps_dev, &P->fx, &P->fy, &P->fz, &P->maxpart, &P->maxout, &P->wt_x,
                    &P->wt_y, &P->wt_z, &P->wt_pe, &P->wt_ph, &P->wt_first, &P->Eo, &P->Ho, &P->errbuf,
                    &P->shifts, &P->yblk, &P->V64, &P->gtw[0], &P->gtw[1], &P->gtw[2], &P->gch[0][0],
                    &P->gch[0][1], &P->gch[1][0], &P->gch[1][1], &P->gch[2][0], &P->gch[2][1], &P->gkn[0][0],
                    &P->gkn[0][1], &P->gkn[1][0], &P->gkn[1][1], &P->gkn[2][0], &P->gkn[2][1]};
  for (DevBuf* b : bufs) b->release();
  tk_resolve(P);
  for (cudaEvent_t e : P->evpool) cudaEventDestroy(e);
  for (int i = 0; i < 2; ++i) {
    if (P->cev[i]) cudaEventDestroy(P->cev[i]);
    if (P->ready[i]) cudaEventDestroy(P->ready[i]);
  }
  if (P->stage_h) cudaFreeHost(P->stage_h);
  if (P->cst) cudaStreamDestroy(P->cst);
  if (P->st) cudaStreamDestroy(P->st);
  delete P;
}

fm_status fm_synchronize(fm_plan* P) {
  if (!P) return fail(FM_ERR_INVALID, "null plan");
  FM_CK(cudaSetDevice(P->desc.device));
  FM_CK(cudaStreamSynchronize(P->st));
  return FM_OK;
}

static void set_scalars(fm_plan* P, double k_bg, double eps_imag, double wavelength) {
  P->k_bg = k_bg;
  P->eps_imag = eps_imag;
  P->wavelength = wavelength;
  P->kref2 = (k_bg > 0) ? k_bg * k_bg : 1.0;
}

fm_status fm_set_potential(fm_plan* P, const double* V, double k_bg, double eps_imag, double wavelength) {
  FM_TRY(check_plan(P, 1, false));
  if (!V) return fail(FM_ERR_INVALID, "null potential");
  if (!(k_bg > 0) || !(eps_imag > 0) || !(wavelength > 0)) return fail(FM_ERR_INVALID, "k_bg, eps_imag, wavelength must be positive");
  set_scalars(P, k_bg, eps_imag, wavelength);
  FM_CK(P->V.ensure((size_t)P->n * P->esz));
  if (P->prec == FM_PREC_F64) FM_TRY(h2d_field<double>(P, V, P->n, 1.0 / P->kref2, P->V.p));
  else FM_TRY(h2d_field<float>(P, V, P->n, 1.0 / P->kref2, P->V.p));
  FM_CK(cudaStreamSynchronize(P->st));
  P->have_pot = true;
  return FM_OK;
}

template <typename R>
static fm_status apply_host(fm_plan* P, int nrhs, const double* x, double* y, int mode, cd alpha, cd beta) {
  const long long cnt = (long long)nrhs * P->M;
  const size_t fbytes = (size_t)cnt * sizeof(cplx<R>);
  FM_CK(P->sbuf.ensure(fbytes));
  FM_CK(P->ebuf.ensure(fbytes));
  EpiParams ep{};
  ep.alpha_re = alpha.real();
  ep.alpha_im = alpha.imag();
  ep.beta_re = beta.real();
  ep.beta_im = beta.imag();
  ep.inv_eps = P->kref2 / P->eps_imag;
  if (mode == 0) {  // Green: input scaled by 1/kref2 so that G' x' = G x
    FM_TRY(h2d_field<R>(P, x, cnt, 1.0 / P->kref2, P->sbuf.p));
    FM_TRY(green_op<R>(P, nrhs, P->sbuf.p, PRO_COPY, nullptr, EPI_STORE, nullptr, nullptr, ep, P->ebuf.p, nullptr));
  } else if (mode == 1) {  // operator
    FM_TRY(h2d_field<R>(P, x, cnt, 1.0, P->sbuf.p));
    if (beta != 0.0) FM_TRY(h2d_field<R>(P, y, cnt, 1.0, P->ebuf.p));
    FM_TRY(green_op<R>(P, nrhs, P->sbuf.p, PRO_V, nullptr, EPI_OP, P->sbuf.p, nullptr, ep, P->ebuf.p, nullptr));
  } else if (mode == 2) {  // curl
    FM_TRY(h2d_field<R>(P, x, cnt, 1.0, P->sbuf.p));
    FM_TRY(curl_batch<R>(P, nrhs, P->sbuf.p, P->ebuf.p, nullptr));
  }
  FM_TRY(d2h_field<R>(P, P->ebuf.p, cnt, 1.0, y));
  return check_device_error(P);
}

fm_status fm_green_apply(fm_plan* P, int nrhs, const double* x, double* y) {
  FM_TRY(check_plan(P, nrhs, true));
  if (!x || !y) return fail(FM_ERR_INVALID, "null buffer");
  return P->prec == FM_PREC_F64 ? apply_host<double>(P, nrhs, x, y, 0, 0.0, 0.0) : apply_host<float>(P, nrhs, x, y, 0, 0.0, 0.0);
}

fm_status fm_apply_operator(fm_plan* P, int nrhs, const double* x, double* y, double ar, double ai, double br, double bi) {
  FM_TRY(check_plan(P, nrhs, true));
  if (!x || !y) return fail(FM_ERR_INVALID, "null buffer");
  return P->prec == FM_PREC_F64 ? apply_host<double>(P, nrhs, x, y, 1, cd(ar, ai), cd(br, bi))
                                : apply_host<float>(P, nrhs, x, y, 1, cd(ar, ai), cd(br, bi));
}

fm_status fm_curl_field(fm_plan* P, int nrhs, const double* E, double* H) {
  FM_TRY(check_plan(P, nrhs, false));
  if (!E || !H) return fail(FM_ERR_INVALID, "null buffer");
  if (!(P->wavelength > 0)) return fail(FM_ERR_INVALID, "wavelength not set (fm_set_potential / fm_build_potential)");
  return P->prec == FM_PREC_F64 ? apply_host<double>(P, nrhs, E, H, 2, 0.0, 0.0) : apply_host<float>(P, nrhs, E, H, 2, 0.0, 0.0);
}

template <typename R>
__global__ void k_precond(long long n, int nb, const cplx<R>* __restrict__ V, double inv_eps, const cplx<R>* __restrict__ x,
                          cplx<R>* __restrict__ y) {
  const long long tot = n * 3 * nb;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    cplx<R> v = V[i % n];
    cplx<R> g = mk(-v.y * (R)inv_eps, v.x * (R)inv_eps);
    y[i] = cmul(g, x[i]);
  }
}

template <typename R>
static fm_status precond_host(fm_plan* P, int nrhs, const double* x, double* y) {
  const long long cnt = (long long)nrhs * P->M;
  FM_CK(P->sbuf.ensure((size_t)cnt * sizeof(cplx<R>)));
  FM_CK(P->ebuf.ensure((size_t)cnt * sizeof(cplx<R>)));
  FM_TRY(h2d_field<R>(P, x, cnt, 1.0, P->sbuf.p));
  k_precond<R><<<1184, 256, 0, P->st>>>(P->n, nrhs, (const cplx<R>*)P->V.p, P->kref2 / P->eps_imag,
                                        (const cplx<R>*)P->sbuf.p, (cplx<R>*)P->ebuf.p);
  FM_CK(cudaGetLastError());
  return d2h_field<R>(P, P->ebuf.p, cnt, 1.0, y);
}

fm_status fm_apply_preconditioner(fm_plan* P, int nrhs, const double* x, double* y) {
  FM_TRY(check_plan(P, nrhs, true));
  if (!x || !y) return fail(FM_ERR_INVALID, "null buffer");
  return P->prec == FM_PREC_F64 ? precond_host<double>(P, nrhs, x, y) : precond_host<float>(P, nrhs, x, y);
}

template <typename R>
static fm_status solve_source_t(fm_plan* P, int nrhs, const double* S, const fm_solve_opts& o, double* E, double* H,
                                fm_solve_info* info) {
  int wave = 1;
  FM_TRY(plan_wave_size<R>(P, nrhs, o, wave));
  bool all_ok = true;
  for (int b0 = 0; b0 < nrhs; b0 += wave) {
    const int nb = std::min(wave, nrhs - b0);
    const long long cnt = (long long)nb * P->M;
    FM_CK(P->sbuf.ensure((size_t)cnt * sizeof(cplx<R>)));
    FM_TRY(h2d_field<R>(P, S + (size_t)b0 * P->M * 2, cnt, 1.0 / P->kref2, P->sbuf.p));
    std::vector<fm_solve_info> inf(nb);
    FM_TRY(solve_core<R>(P, nb, o, inf));
    FM_TRY(d2h_field<R>(P, P->xbuf.p, cnt, 1.0, E + (size_t)b0 * P->M * 2));
    FM_TRY(d2h_field<R>(P, P->ebuf.p, cnt, 1.0, H + (size_t)b0 * P->M * 2));
    for (int b = 0; b < nb; ++b) {
      if (info) info[b0 + b] = inf[b];
      all_ok &= inf[b].solved != 0;
    }
  }
  if (!all_ok) return fail(FM_NOT_CONVERGED, "iteration limit reached before the tolerance was met");
  return FM_OK;
}

fm_status fm_solve_source(fm_plan* P, int nrhs, const double* S, const fm_solve_opts* opts, double* E, double* H,
                          fm_solve_info* info) {
  FM_TRY(check_plan(P, nrhs, true));
  FM_TRY(validate_opts(opts));
  if (!S || !E || !H) return fail(FM_ERR_INVALID, "null buffer");
  return P->prec == FM_PREC_F64 ? solve_source_t<double>(P, nrhs, S, *opts, E, H, info)
                                : solve_source_t<float>(P, nrhs, S, *opts, E, H, info);
}

template <typename R>
static fm_status build_potential_t(fm_plan* P, const double* eps, double eps_bg, double wl, const double* fx,
                                   const double* fy, const double* fz, int itmax, fm_potential_info* info) {
  const long long g = (long long)P->pi.gx * P->pi.gy * P->pi.gz;
  FM_CK(P->eps_dev.ensure((size_t)g * sizeof(double2)));
  FM_CK(cudaMemcpyAsync(P->eps_dev.p, eps, (size_t)g * sizeof(double2), cudaMemcpyHostToDevice, P->st));
  {
    // NaN/Inf in the permittivity would propagate silently (fmax ignores NaN): reject it here
    FM_CK(P->maxout.ensure(sizeof(double) + sizeof(unsigned) + sizeof(unsigned long long) + 8));
    unsigned long long* bad = (unsigned long long*)((char*)P->maxout.p + 16);
    FM_CK(cudaMemsetAsync(bad, 0, sizeof(unsigned long long), P->st));
    k_count_nonfinite<double><<<592, 256, 0, P->st>>>(g, (const double2*)P->eps_dev.p, bad);
    FM_CK(cudaGetLastError());
    unsigned long long nbad = 0;
    FM_CK(cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
    if (nbad) return fail(FM_ERR_NONFINITE, "permittivity contains NaN or Inf");
  }
  const int nb = 592;
  FM_CK(P->maxpart.ensure(nb * sizeof(double)));
  unsigned* cnt = (unsigned*)((char*)P->maxout.p + sizeof(double));
  FM_CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned), P->st));
  const double k_bg = 2.0 * M_PI * std::sqrt(eps_bg) / wl;
  const double k2 = k_bg * k_bg;
  k_potential_max<<<nb, 256, 0, P->st>>>(g, (const double2*)P->eps_dev.p, eps_bg, k2, (double*)P->maxpart.p,
                                          (double*)P->maxout.p, cnt);
  FM_CK(cudaGetLastError());
  double vmax = 0.0;
  FM_CK(cudaMemcpyAsync(&vmax, P->maxout.p, sizeof(double), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  if (!std::isfinite(vmax)) return fail(FM_ERR_NONFINITE, "non-finite permittivity");
  // with padding the zero-padded region also enters the maximum (|0| never exceeds it)
  const double eps_imag = std::max(std::pow(2.0, -20), vmax * 1.01);
  set_scalars(P, k_bg, eps_imag, wl);
  const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
  DevBuf* fb[3] = {&P->fx, &P->fy, &P->fz};
  const double* fh[3] = {fx, fy, fz};
  for (int a = 0; a < 3; ++a) {
    std::vector<double> ones(n3[a], 1.0);
    FM_CK(fb[a]->ensure(n3[a] * sizeof(double)));
    FM_CK(cudaMemcpyAsync(fb[a]->p, fh[a] ? fh[a] : ones.data(), n3[a] * sizeof(double), cudaMemcpyHostToDevice, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
  }
  FM_CK(P->V.ensure((size_t)P->n * P->esz));
  k_potential_build<R><<<1184, 256, 0, P->st>>>(P->pi, (const double2*)P->eps_dev.p, eps_bg, k2, eps_imag,
                                                (const double*)P->fx.p, (const double*)P->fy.p, (const double*)P->fz.p,
                                                1.0 / P->kref2, (cplx<R>*)P->V.p);
  FM_CK(cudaGetLastError());
  int bornmax;
  if (itmax < 0) {
    const double steps = std::abs(2.0 * k_bg / eps_imag);
    double ext = 0.0;
    for (int a = 0; a < 3; ++a) ext += std::pow(n3[a] * P->desc.resolution[a], 2);
    ext = std::sqrt(ext);
    const int opt = (int)std::ceil(ext / steps / 2.0 + 1.0) * 2;
    bornmax = opt * std::abs(itmax);
  } else {
    bornmax = itmax;
  }
  P->bornmax = bornmax;
  FM_CK(cudaStreamSynchronize(P->st));
  P->have_pot = true;
  if (info) {
    info->eps_imag = eps_imag;
    info->k_bg = k_bg;
    info->bornmax = bornmax;
  }
  return FM_OK;
}

fm_status fm_build_potential(fm_plan* P, const double* eps, double eps_bg, double wl, const double* fx, const double* fy,
                             const double* fz, int itmax, fm_potential_info* info) {
  FM_TRY(check_plan(P, 1, false));
  if (!eps) return fail(FM_ERR_INVALID, "null permittivity");
  if (!(eps_bg > 0)) return fail(FM_ERR_INVALID, "permittivity_bg must be positive");
  if (!(wl > 0)) return fail(FM_ERR_INVALID, "wavelength must be positive");
  return P->prec == FM_PREC_F64 ? build_potential_t<double>(P, eps, eps_bg, wl, fx, fy, fz, itmax, info)
                                : build_potential_t<float>(P, eps, eps_bg, wl, fx, fy, fz, itmax, info);
}

// Plane-wave tables (FP64) of one source, following generate_incident_field
// (sources.jl): per-axis phase tables exp(i k_b k_d r_d) over the padded axis
// (source amplitude and phase folded into the z table) and the E and H
// polarisations.  tx/ty/tz have nx/ny/nz entries, pe/ph three each.
static fm_status wave_tables(const fm_plan* P, const fm_plane_wave& w, double eps_bg, double2* tx, double2* ty,
                             double2* tz, double2* pe, double2* ph) {
  const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
  const int g3[3] = {P->pi.gx, P->pi.gy, P->pi.gz};
  const int p3[3] = {P->pi.px, P->pi.py, P->pi.pz};
  if (!(w.wavelength > 0)) return fail(FM_ERR_INVALID, "wavelength must be positive");
  if (!(w.amplitude >= 0)) return fail(FM_ERR_INVALID, "amplitude must be non-negative");
  const double k0 = 2.0 * M_PI / w.wavelength;
  const double kb = k0 * std::sqrt(eps_bg);
  double kn = std::sqrt(w.k_vector[0] * w.k_vector[0] + w.k_vector[1] * w.k_vector[1] + w.k_vector[2] * w.k_vector[2]);
  if (!(std::abs(kn - 1.0) < 1e-10)) return fail(FM_ERR_INVALID, "k_vector must be normalized (|k| = 1)");
  double kh[3];
  for (int a = 0; a < 3; ++a) kh[a] = w.k_vector[a] / kn;
  cd p[3];
  for (int a = 0; a < 3; ++a) p[a] = cd(w.polarization[2 * a], w.polarization[2 * a + 1]);
  cd edotk = std::conj(p[0]) * kh[0] + std::conj(p[1]) * kh[1] + std::conj(p[2]) * kh[2];
  if (!(std::abs(edotk.real()) < 1e-10)) return fail(FM_ERR_INVALID, "polarization must be transverse to k_vector");
  double pn = std::sqrt(std::norm(p[0]) + std::norm(p[1]) + std::norm(p[2]));
  cd e0[3];
  for (int a = 0; a < 3; ++a) e0[a] = p[a] / pn;
  cd d = std::conj(e0[0]) * kh[0] + std::conj(e0[1]) * kh[1] + std::conj(e0[2]) * kh[2];
  cd ep[3];
  for (int a = 0; a < 3; ++a) ep[a] = e0[a] - d * kh[a];
  double en = std::sqrt(std::norm(ep[0]) + std::norm(ep[1]) + std::norm(ep[2]));
  for (int a = 0; a < 3; ++a) ep[a] /= en;
  const double zimp = 377.0 / std::sqrt(eps_bg);
  cd hp[3] = {(kh[1] * ep[2] - kh[2] * ep[1]) / zimp, (kh[2] * ep[0] - kh[0] * ep[2]) / zimp,
              (kh[0] * ep[1] - kh[1] * ep[0]) / zimp};
  for (int a = 0; a < 3; ++a) {
    pe[a] = make_double2(ep[a].real(), ep[a].imag());
    ph[a] = make_double2(hp[a].real(), hp[a].imag());
  }
  double2* tabs[3] = {tx, ty, tz};
  for (int a = 0; a < 3; ++a) {
    const double center = (g3[a] - 1) * P->desc.resolution[a] / 2.0;
    for (int i = 0; i < n3[a]; ++i) {
      const double r = (double)(i - p3[a]) * P->desc.resolution[a] - center;
      cd v = std::exp(cd(0.0, kb * kh[a] * r));
      if (a == 2) v *= w.amplitude * std::exp(cd(0.0, w.phase));
      tabs[a][i] = make_double2(v.real(), v.imag());
    }
  }
  return FM_OK;
}

// plane-wave tables of nrhs right-hand sides (first[] gives each RHS's source range)
static fm_status upload_waves(fm_plan* P, int nrhs, const int* first, const fm_plane_wave* src, double eps_bg) {
  const int ns = first[nrhs];
  const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
  std::vector<double2> tx((size_t)ns * n3[0]), ty((size_t)ns * n3[1]), tz((size_t)ns * n3[2]), pe(ns * 3), ph(ns * 3);
  for (int s = 0; s < ns; ++s)
    FM_TRY(wave_tables(P, src[s], eps_bg, &tx[(size_t)s * n3[0]], &ty[(size_t)s * n3[1]], &tz[(size_t)s * n3[2]],
                       &pe[s * 3], &ph[s * 3]));
  auto up = [&](DevBuf& b, const void* h, size_t bytes) -> fm_status {
    FM_CK(b.ensure(std::max<size_t>(bytes, 16)));
    FM_CK(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, P->st));
    return FM_OK;
  };
  FM_TRY(up(P->wt_x, tx.data(), tx.size() * sizeof(double2)));
  FM_TRY(up(P->wt_y, ty.data(), ty.size() * sizeof(double2)));
  FM_TRY(up(P->wt_z, tz.data(), tz.size() * sizeof(double2)));
  FM_TRY(up(P->wt_pe, pe.data(), pe.size() * sizeof(double2)));
  FM_TRY(up(P->wt_ph, ph.data(), ph.size() * sizeof(double2)));
  FM_TRY(up(P->wt_first, first, (nrhs + 1) * sizeof(int)));
  FM_CK(cudaStreamSynchronize(P->st));
  return FM_OK;
}

// ---------------------------------------------------------------------------
// Output copies.  The caller's E/H buffers are ordinary (pageable) host memory.  A worker thread copies each
// finished wave device -> pinned staging chunk (copy stream) -> caller buffer (host threads), so the copy of
// wave i runs while wave i+1 computes, and the host-side page faults of a fresh destination are taken by
// several threads.  The solve thread's own small reads stay on the compute stream.
// ---------------------------------------------------------------------------
constexpr size_t OUT_CHUNK = (size_t)32 << 20;

static fm_status ensure_copier(fm_plan* P) {
  if (!P->cst) FM_CK(cudaStreamCreateWithFlags(&P->cst, cudaStreamNonBlocking));
  if (!P->stage_h) FM_CK(cudaHostAlloc(&P->stage_h, 2 * OUT_CHUNK, cudaHostAllocDefault));
  for (int i = 0; i < 2; ++i) {
    if (!P->cev[i]) FM_CK(cudaEventCreateWithFlags(&P->cev[i], cudaEventDisableTiming));
    if (!P->ready[i]) FM_CK(cudaEventCreateWithFlags(&P->ready[i], cudaEventDisableTiming));
  }
  return FM_OK;
}

static void host_copy(char* dst, const char* src, size_t n) {
  // the first write to a fresh pageable destination faults its pages in: several threads take the faults in parallel
  static const int NT = std::max(2, std::min(8, (int)std::thread::hardware_concurrency() / 2));
  if (n < ((size_t)4 << 20)) {
    std::memcpy(dst, src, n);
    return;
  }
  const size_t part = ((n + NT - 1) / NT + 63) & ~(size_t)63;
  std::vector<std::thread> th;
  th.reserve(NT - 1);
  for (int i = 1; i < NT; ++i) {
    const size_t a = std::min(n, part * i), b = std::min(n, part * (i + 1));
    if (b > a) th.emplace_back([=] { std::memcpy(dst + a, src + a, b - a); });
  }
  std::memcpy(dst, src, std::min(n, part));
  for (auto& t : th) t.join();
}

// Copies `bytes` from each of de, dh (device) to E, H (host) once event ready[slot] has completed.
static cudaError_t copy_out(fm_plan* P, int slot, const void* de, const void* dh, void* E, void* H, size_t bytes) {
  cudaError_t e = cudaSetDevice(P->desc.device);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(P->cst, P->ready[slot], 0);
  char* stage = (char*)P->stage_h;
  char* pdst[2] = {nullptr, nullptr};
  size_t pn[2] = {0, 0};
  const char* src[2] = {(const char*)de, (const char*)dh};
  char* dst[2] = {(char*)E, (char*)H};
  auto drain = [&](int s) {
    if (!pdst[s]) return;
    const cudaError_t e2 = cudaEventSynchronize(P->cev[s]);
    if (e2 == cudaSuccess) host_copy(pdst[s], stage + s * OUT_CHUNK, pn[s]);
    else if (e == cudaSuccess) e = e2;
    pdst[s] = nullptr;
  };
  int i = 0;
  for (int f = 0; f < 2 && e == cudaSuccess; ++f)
    for (size_t off = 0; off < bytes && e == cudaSuccess; off += OUT_CHUNK, ++i) {
      const int s = i & 1;
      drain(s);
      if (e != cudaSuccess) break;
      const size_t n = std::min(OUT_CHUNK, bytes - off);
      e = cudaMemcpyAsync(stage + s * OUT_CHUNK, src[f] + off, n, cudaMemcpyDeviceToHost, P->cst);
      if (e == cudaSuccess) e = cudaEventRecord(P->cev[s], P->cst);
      if (e == cudaSuccess) {
        pdst[s] = dst[f] + off;
        pn[s] = n;
      }
    }
  drain(i & 1);
  drain((i + 1) & 1);
  return e;
}

template <typename R>
static fm_status solve_waves_t(fm_plan* P, int nrhs, const int* first, const fm_plane_wave* src, double eps_bg,
                               const fm_solve_opts& o, double* E, double* H, fm_solve_info* info) {
  int wave = 1;
  FM_TRY(plan_wave_size<R>(P, nrhs, o, wave));
  const long long g = (long long)P->pi.gx * P->pi.gy * P->pi.gz;
  const bool keep = (E == nullptr);
  // host outputs: two device output slots when there is more than one wave (wave i copied while i+1 runs)
  const int slots = (!keep && nrhs > wave) ? 2 : 1;
  if (keep) {
    FM_CK(P->Eo.ensure((size_t)nrhs * 3 * g * sizeof(double2)));
    FM_CK(P->Ho.ensure((size_t)nrhs * 3 * g * sizeof(double2)));
  } else {
    FM_CK(P->Eo.ensure((size_t)slots * wave * 3 * g * sizeof(double2)));
    FM_CK(P->Ho.ensure((size_t)slots * wave * 3 * g * sizeof(double2)));
    FM_TRY(ensure_copier(P));
  }
  std::future<cudaError_t> pend[2];
  bool all_ok = true;
  for (int b0 = 0, wi = 0; b0 < nrhs; b0 += wave, ++wi) {
    const int nb = std::min(wave, nrhs - b0);
    const int slot = wi % slots;
    std::vector<int> f(nb + 1);
    for (int b = 0; b <= nb; ++b) f[b] = first[b0 + b] - first[b0];
    FM_TRY(upload_waves(P, nb, f.data(), src + first[b0], eps_bg));
    FM_CK(P->sbuf.ensure((size_t)nb * P->M * sizeof(cplx<R>)));
    WaveTabs wt{(const double2*)P->wt_x.p, (const double2*)P->wt_y.p, (const double2*)P->wt_z.p,
                (const double2*)P->wt_pe.p, (const double2*)P->wt_ph.p, (const int*)P->wt_first.p};
    FM_TRACK(P, KC_SETUP, (double)nb * P->M * sizeof(cplx<R>) + (double)P->n * sizeof(cplx<R>),
             (k_source_term<R><<<dim3(296, nb), 256, 0, P->st>>>(P->pi, nb, wt, (const cplx<R>*)P->V.p,
                                                                 P->eps_imag / P->kref2, (cplx<R>*)P->sbuf.p, nullptr)));
    FM_CK(cudaGetLastError());
    std::vector<fm_solve_info> inf(nb);
    FM_TRY(solve_core<R>(P, nb, o, inf));
    if (pend[slot].valid()) FM_CK(pend[slot].get());  // the slot's previous wave has reached the host
    const size_t oo = keep ? (size_t)b0 * 3 * g : (size_t)slot * wave * 3 * g;
    double2* eo = (double2*)P->Eo.p + oo;
    double2* ho = (double2*)P->Ho.p + oo;
    FM_TRACK(P, KC_SETUP, (double)nb * 3 * g * (2 * sizeof(cplx<R>) + 2 * sizeof(double2)),
             (k_assemble<R><<<dim3(296, nb), 256, 0, P->st>>>(P->pi, nb, wt, (const cplx<R>*)P->xbuf.p,
                                                              (const cplx<R>*)P->ebuf.p, eo, ho)));
    FM_CK(cudaGetLastError());
    if (!keep) {
      FM_CK(cudaEventRecord(P->ready[slot], P->st));
      pend[slot] = std::async(std::launch::async, copy_out, P, slot, (const void*)eo, (const void*)ho,
                              (void*)(E + (size_t)b0 * 3 * g * 2), (void*)(H + (size_t)b0 * 3 * g * 2),
                              (size_t)nb * 3 * g * sizeof(double2));
    }
    FM_CK(cudaStreamSynchronize(P->st));
    tk_resolve(P);
    for (int b = 0; b < nb; ++b) {
      if (info) info[b0 + b] = inf[b];
      all_ok &= inf[b].solved != 0;
    }
  }
  for (auto& f : pend)
    if (f.valid()) FM_CK(f.get());
  P->out_nrhs = keep ? nrhs : 0;
  if (!all_ok) return fail(FM_NOT_CONVERGED, "iteration limit reached before the tolerance was met");
  return FM_OK;
}

fm_status fm_solve_plane_waves(fm_plan* P, int nrhs, const int* first, const fm_plane_wave* sources, double eps_bg,
                               const fm_solve_opts* opts, double* E, double* H, fm_solve_info* info) {
  FM_TRY(check_plan(P, nrhs, true));
  FM_TRY(validate_opts(opts));
  if (!first || !sources) return fail(FM_ERR_INVALID, "null sources");
  if ((E == nullptr) != (H == nullptr)) return fail(FM_ERR_INVALID, "E_out and H_out must both be set or both be NULL");
  if (first[0] != 0) return fail(FM_ERR_INVALID, "first[0] must be 0");
  for (int b = 0; b < nrhs; ++b)
    if (first[b + 1] <= first[b]) return fail(FM_ERR_INVALID, "sources vector cannot be empty");
  for (int b = 0; b < nrhs; ++b) {
    for (int s = first[b] + 1; s < first[b + 1]; ++s)
      if (sources[s].wavelength != sources[first[b]].wavelength)
        return fail(FM_ERR_INVALID, "All sources must have the same wavelength for coherent superposition");
    if (std::abs(sources[first[b]].wavelength - P->wavelength) > 1e-12 * P->wavelength)
      return fail(FM_ERR_INVALID, "source wavelength differs from the wavelength of the potential");
  }
  if (!(eps_bg > 0)) return fail(FM_ERR_INVALID, "permittivity_bg must be positive");
  return P->prec == FM_PREC_F64 ? solve_waves_t<double>(P, nrhs, first, sources, eps_bg, *opts, E, H, info)
                                : solve_waves_t<float>(P, nrhs, first, sources, eps_bg, *opts, E, H, info);
}

fm_status fm_copy_fields(fm_plan* P, int nrhs, double* E, double* H) {
  FM_TRY(check_plan(P, nrhs, false));
  if (!E || !H) return fail(FM_ERR_INVALID, "null buffer");
  if (nrhs > P->out_nrhs) return fail(FM_ERR_INVALID, "fewer fields are resident than requested");
  const long long g = (long long)P->pi.gx * P->pi.gy * P->pi.gz;
  FM_CK(cudaMemcpyAsync(E, P->Eo.p, (size_t)nrhs * 3 * g * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaMemcpyAsync(H, P->Ho.p, (size_t)nrhs * 3 * g * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  return FM_OK;
}


fm_status fm_set_profiling(fm_plan* P, int on) {
  if (!P) return fail(FM_ERR_INVALID, "null plan");
  FM_CK(cudaSetDevice(P->desc.device));
  FM_CK(cudaStreamSynchronize(P->st));
  tk_resolve(P);
  P->prof = on != 0;
  for (int i = 0; i < KC_N; ++i) {
    P->launches[i] = 0;
    P->kms[i] = 0;
    P->kbytes[i] = 0;
  }
  P->total_launches = 0;
  return FM_OK;
}

int fm_kernel_stats(fm_plan* P, fm_kernel_stat* out, int max) {
  if (!P) return -1;
  cudaSetDevice(P->desc.device);
  cudaStreamSynchronize(P->st);
  tk_resolve(P);
  int n = 0;
  for (int i = 0; i < KC_N && n < max; ++i, ++n) {
    std::snprintf(out[n].name, sizeof(out[n].name), "%s", kcls_name[i]);
    out[n].launches = P->launches[i];
    out[n].ms = P->kms[i];
    out[n].bytes = P->kbytes[i];
  }
  return n;
}

long long fm_launch_count(fm_plan* P) { return P ? P->total_launches : -1; }

void* fm_stream(fm_plan* P) { return P ? (void*)P->st : nullptr; }

fm_status fm_plan_set_tuning(fm_plan* P, int knob, int value) {
  if (!P) return fail(FM_ERR_INVALID, "null plan");
  FM_CK(cudaSetDevice(P->desc.device));
  FM_CK(cudaStreamSynchronize(P->st));
  switch (knob) {
    case FM_TUNE_Y_TMA:
    case FM_TUNE_Z_TMA:
      if (value != 0 && value != 1) return fail(FM_ERR_INVALID, "TMA tuning value must be 0 or 1");
      (knob == FM_TUNE_Y_TMA ? P->tma_y : P->tma_z) = value != 0;
      return FM_OK;
    case FM_TUNE_TMA_CTAS_PER_SM:
      if (value < 0 || value > 32) return fail(FM_ERR_INVALID, "TMA CTAs per SM must be 0..32");
      P->dims.tma_ctas = value;
      return FM_OK;
    case FM_TUNE_ROW_THREADS:
      if (value != 128 && value != 256) return fail(FM_ERR_INVALID, "row-pass threads must be 128 or 256");
      P->dims.row_threads = value;
      return FM_OK;
    case FM_TUNE_WAVE_RHS:
      if (value < 0) return fail(FM_ERR_INVALID, "right-hand sides per wave must be >= 0");
      P->wave_rhs = value;
      return FM_OK;
    case FM_TUNE_BLOCK_DOT:
      if (value != 0 && value != 1) return fail(FM_ERR_INVALID, "block-dot tuning value must be 0 or 1");
      P->bd_bulk = value != 0;
      return FM_OK;
    default:
      return fail(FM_ERR_INVALID, "unknown tuning knob");
  }
}

fm_status fm_plan_get_tuning(fm_plan* P, int knob, int* value) {
  if (!P || !value) return fail(FM_ERR_INVALID, "null argument");
  switch (knob) {
    case FM_TUNE_Y_TMA: *value = P->tma_y ? 1 : 0; return FM_OK;
    case FM_TUNE_Z_TMA: *value = P->tma_z ? 1 : 0; return FM_OK;
    case FM_TUNE_TMA_CTAS_PER_SM: *value = P->dims.tma_ctas; return FM_OK;
    case FM_TUNE_ROW_THREADS: *value = P->dims.row_threads; return FM_OK;
    case FM_TUNE_WAVE_RHS: *value = P->wave_rhs; return FM_OK;
    case FM_TUNE_BLOCK_DOT: *value = P->bd_bulk ? 1 : 0; return FM_OK;
    default: return fail(FM_ERR_INVALID, "unknown tuning knob");
  }
}

// ===========================================================================
// Slot engine: continuous batching of independent right-hand sides.
//
// An engine owns S slots on one plan.  A slot holds one right-hand side (one
// plane wave on one permittivity) with its own potential, eps_imag, Krylov
// basis (slot-major: U[(i*S + s)*M]) and GMRES state.  Each fm_engine_step
//   1. admits queued right-hand sides into free slots (potential, plane-wave
//      tables, source term, b = G S, x = b);
//   2. forms r0 = M^{-1}(b - A x) for slots just admitted or restarted;
//   3. runs ONE GMRES iteration on every running slot in shared launches
//      (each slot at its own inner index j: per-slot vector pointers and basis
//      sizes);
//   4. adds the Krylov correction to x for slots whose cycle ended (stop or
//      restart after `basis` inner iterations);
//   5. finishes the stopped slots (magnetic field, incident addition, crop,
//      copy to the caller's host buffers).
// A right-hand side follows exactly the iteration of the batched GMRES with
// restart = basis (full GMRES when its iteration limit fits the basis), so its
// result does not depend on the other slots.  All requests of an engine share
// wavelength and background permittivity.
// ===========================================================================
struct EngineUnit {  // one queued right-hand side
  long long req;
  int rhs;                                        // index within its request
  std::shared_ptr<std::vector<double2>> eps_sh;   // unpadded permittivity, shared by the request's units
  fm_plane_wave src;
  double tol;
  int itmax_setting;
  double* E_out;  // host, (gx,gy,gz,3) FP64 complex for this RHS
  double* H_out;
};

enum { SL_FREE = 0, SL_RUN = 1, SL_STOP = 2, SL_RESTART = 3, SL_RESIDUAL = 4 };

struct EngineSlot {
  int state = SL_FREE;
  bool fresh = false;  // admitted, residual not formed yet
  EngineUnit u;
  int j = 0, inner = 0, iters = 0, maxiters = 100;
  double beta = 0, eps = 0, rnorm = 0, eps_imag = 0, beta0 = 0;
  bool solved = false;
  std::vector<double> c;
  std::vector<cd> sn, z;
  std::vector<std::vector<cd>> R;
};

struct fm_engine {
  fm_plan* P = nullptr;
  int S = 0, mem = 100;
  double wavelength = 0, eps_bg = 0;
  int ortho = FM_ORTHO_CGS;
  DevBuf U, X, Bv, Sb, Hb, Vs, ksq, ieps, scale, act, kb, tabs, Eo, Ho, wt_x, wt_y, wt_z, wt_pe, wt_ph, wt_first,
      epsd, maxp, maxo;
  std::vector<EngineSlot> slots;
  std::deque<EngineUnit> queue;
  std::mutex mu;
  std::vector<double> sch;  // host copy of the basis scales [(mem+1) x S]
  struct Done {
    long long req;
    int rhs;
    fm_solve_info info;
  };
  std::deque<Done> done;
};

long long fm_engine_slot_bytes(const fm_plan_desc* d, int basis) {
  if (!d) return -1;
  long long n = 1, g = 1;
  for (int a = 0; a < 3; ++a) {
    n *= (long long)(d->grid[a] + 2 * d->pad[a]);
    g *= d->grid[a];
  }
  const long long esz = d->precision == FM_PREC_F64 ? 16 : 8;
  // basis + x + b + source + curl + two pass temporaries (3-component fields), potential, FP64 outputs
  return 3 * n * esz * (basis + 1 + 6) + n * esz + 2 * 3 * g * 16;
}

fm_status fm_engine_create(fm_plan* P, int slots, int basis, double wavelength, double eps_bg, const double* fx,
                           const double* fy, const double* fz, int ortho, fm_engine** out) {
  if (!P || !out || slots < 1 || basis < 1) return fail(FM_ERR_INVALID, "fm_engine_create: bad argument");
  *out = nullptr;
  if (basis + 1 > KV_KMAX) return fail(FM_ERR_UNSUPPORTED, "Krylov basis larger than 127 vectors");
  if (!(wavelength > 0) || !(eps_bg > 0)) return fail(FM_ERR_INVALID, "wavelength and permittivity_bg must be positive");
  if (ortho != FM_ORTHO_CGS && ortho != FM_ORTHO_CGS2) return fail(FM_ERR_INVALID, "the engine runs CGS or CGS2");
  FM_CK(cudaSetDevice(P->desc.device));
  fm_engine* E = new fm_engine();
  E->P = P;
  E->S = slots;
  E->mem = basis;
  E->ortho = ortho;
  E->wavelength = wavelength;
  E->eps_bg = eps_bg;
  const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
  {
    const double* fh[3] = {fx, fy, fz};
    DevBuf* fb[3] = {&P->fx, &P->fy, &P->fz};
    for (int a = 0; a < 3; ++a) {
      std::vector<double> f(n3[a], 1.0);
      if (fh[a]) f.assign(fh[a], fh[a] + n3[a]);
      cudaError_t e = fb[a]->ensure(n3[a] * sizeof(double));
      if (e == cudaSuccess) e = cudaMemcpy(fb[a]->p, f.data(), n3[a] * sizeof(double), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        delete E;
        return fail(FM_ERR_CUDA, std::string("engine filters: ") + cudaGetErrorString(e));
      }
    }
  }
  // plan scalars: every request shares k_bg and the wavelength; eps_imag is per slot
  set_scalars(P, 2.0 * M_PI * std::sqrt(eps_bg) / wavelength, 1.0, wavelength);
  const size_t M = (size_t)P->M, esz = P->esz, n = (size_t)P->n, S = (size_t)slots;
  const long long g = (long long)P->pi.gx * P->pi.gy * P->pi.gz;
  cudaError_t e = cudaSuccess;
  auto al = [&](DevBuf& b, size_t bytes) {
    if (e == cudaSuccess) e = b.ensure(std::max<size_t>(bytes, 16));
  };
  al(E->U, (size_t)(basis + 1) * S * M * esz);
  al(E->X, S * M * esz);
  al(E->Bv, S * M * esz);
  al(E->Sb, S * M * esz);
  al(E->Hb, S * M * esz);
  al(E->Vs, S * n * esz);
  al(E->ksq, S * sizeof(double));
  al(E->ieps, S * sizeof(double));
  al(E->scale, S * sizeof(double));
  al(E->act, S * sizeof(int));
  al(E->kb, S * sizeof(int));
  al(E->tabs, 2 * S * sizeof(void*));
  al(E->Eo, S * 3 * g * sizeof(double2));
  al(E->Ho, S * 3 * g * sizeof(double2));
  al(E->wt_x, S * n3[0] * sizeof(double2));
  al(E->wt_y, S * n3[1] * sizeof(double2));
  al(E->wt_z, S * n3[2] * sizeof(double2));
  al(E->wt_pe, S * 3 * sizeof(double2));
  al(E->wt_ph, S * 3 * sizeof(double2));
  al(E->wt_first, (S + 1) * sizeof(int));
  al(E->epsd, (size_t)g * sizeof(double2));
  al(E->maxp, 592 * sizeof(double));
  al(E->maxo, 64);
  if (e == cudaSuccess) e = P->t1.ensure(S * M * esz);
  if (e == cudaSuccess) e = P->t2.ensure(S * M * esz);
  if (e == cudaSuccess) e = P->scale.ensure((size_t)(KV_KMAX + 1) * S * sizeof(double));
  if (e == cudaSuccess) e = P->coef.ensure((size_t)(KV_KMAX + 1) * S * sizeof(double2));
  std::vector<int> first(S + 1);
  for (size_t s = 0; s <= S; ++s) first[s] = (int)s;
  std::vector<double> zero(S, 0.0);
  if (e == cudaSuccess) e = cudaMemcpy(E->wt_first.p, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(E->maxo.p, 0, 64);
  if (e == cudaSuccess) e = cudaMemcpy(E->ksq.p, zero.data(), S * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(E->ieps.p, zero.data(), S * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    fm_engine_destroy(E);
    return fail(e == cudaErrorMemoryAllocation ? FM_ERR_OOM : FM_ERR_CUDA, std::string("engine allocation: ") +
                                                                              cudaGetErrorString(e));
  }
  fm_status st = ensure_reduce(P, slots, basis + 1);
  if (st != FM_OK) {
    fm_engine_destroy(E);
    return st;
  }
  E->slots.resize(S);
  E->sch.assign((size_t)(basis + 2) * S, 0.0);
  *out = E;
  return FM_OK;
}

void fm_engine_destroy(fm_engine* E) {
  if (!E) return;
  cudaSetDevice(E->P->desc.device);
  cudaStreamSynchronize(E->P->st);
  DevBuf* b[] = {&E->U, &E->X, &E->Bv, &E->Sb, &E->Hb, &E->Vs, &E->ksq, &E->ieps, &E->scale, &E->act, &E->kb,
                 &E->tabs, &E->Eo, &E->Ho, &E->wt_x, &E->wt_y, &E->wt_z, &E->wt_pe, &E->wt_ph, &E->wt_first,
                 &E->epsd, &E->maxp, &E->maxo};
  for (DevBuf* x : b) x->release();
  delete E;
}

fm_status fm_engine_submit(fm_engine* E, long long request_id, const double* eps, int nrhs,
                           const fm_plane_wave* sources, double tolerance, int iterations_max, double* E_out,
                           double* H_out) {
  if (!E || !eps || !sources || !E_out || !H_out || nrhs < 1) return fail(FM_ERR_INVALID, "fm_engine_submit: bad argument");
  if (!(tolerance >= 0 && tolerance <= 1)) return fail(FM_ERR_INVALID, "tolerance must be in [0, 1]");
  const fm_plan* P = E->P;
  const long long g = (long long)P->pi.gx * P->pi.gy * P->pi.gz;
  auto sh = std::make_shared<std::vector<double2>>((const double2*)eps, (const double2*)eps + g);
  for (long long i = 0; i < g; ++i)
    if (!std::isfinite((*sh)[i].x) || !std::isfinite((*sh)[i].y))
      return fail(FM_ERR_NONFINITE, "permittivity contains NaN or Inf");
  {
    // validate every source now (the same checks as the batched path), so a bad request never takes a slot
    std::vector<double2> tx(P->dims.nx), ty(P->dims.ny), tz(P->dims.nz), pe(3), ph(3);
    for (int r = 0; r < nrhs; ++r) {
      if (std::abs(sources[r].wavelength - E->wavelength) > 1e-12 * E->wavelength)
        return fail(FM_ERR_INVALID, "all requests of an engine share its wavelength");
      FM_TRY(wave_tables(P, sources[r], E->eps_bg, tx.data(), ty.data(), tz.data(), pe.data(), ph.data()));
    }
  }
  std::lock_guard<std::mutex> lk(E->mu);
  for (int r = 0; r < nrhs; ++r) {
    EngineUnit u;
    u.req = request_id;
    u.rhs = r;
    u.eps_sh = sh;
    u.src = sources[r];
    u.tol = tolerance;
    u.itmax_setting = iterations_max;
    u.E_out = E_out + (size_t)r * 3 * g * 2;
    u.H_out = H_out + (size_t)r * 3 * g * 2;
    E->queue.push_back(std::move(u));
  }
  return FM_OK;
}

fm_status fm_engine_status(fm_engine* E, int* running, int* queued) {
  if (!E) return fail(FM_ERR_INVALID, "null engine");
  std::lock_guard<std::mutex> lk(E->mu);
  int r = 0;
  for (auto& s : E->slots) r += s.state != SL_FREE;
  if (running) *running = r;
  if (queued) *queued = (int)E->queue.size();
  return FM_OK;
}

// Bornmax of a right-hand side (convergent_born.jl:653-660)
static int engine_bornmax(const fm_plan* P, double eps_imag, int itmax_setting) {
  if (itmax_setting >= 0) return itmax_setting;
  const double steps = std::abs(2.0 * P->k_bg / eps_imag);
  const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
  double ext = 0.0;
  for (int a = 0; a < 3; ++a) ext += std::pow(n3[a] * P->desc.resolution[a], 2);
  return (int)std::ceil(std::sqrt(ext) / steps / 2.0 + 1.0) * 2 * std::abs(itmax_setting);
}

template <typename R>
static fm_status engine_step_t(fm_engine* E) {
  using T = cplx<R>;
  fm_plan* P = E->P;
  const int S = E->S;
  const size_t M = (size_t)P->M, n = (size_t)P->n;
  const long long g = (long long)P->pi.gx * P->pi.gy * P->pi.gz;
  const double kref2 = P->kref2, k2 = P->k_bg * P->k_bg;
  const double btol = std::pow(2.220446049250313e-16, 0.75);
  T* U = (T*)E->U.p;
  int* act = (int*)E->act.p;
  std::vector<int> acth(S, 0);
  // mark the slots in `states` active; returns their indices
  auto select = [&](std::initializer_list<int> states) {
    std::vector<int> v;
    for (int s = 0; s < S; ++s) {
      acth[s] = 0;
      for (int q : states)
        if (E->slots[s].state == q) acth[s] = 1;
      if (acth[s]) v.push_back(s);
    }
    return v;
  };
  auto upload_act = [&]() -> fm_status {
    FM_CK(cudaMemcpyAsync(act, acth.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
    return FM_OK;
  };
  RhsCtx rc;
  rc.V = E->Vs.p;
  rc.vstride = (long long)n;
  rc.ksq_im_b = (const double*)E->ksq.p;
  rc.inv_eps_b = (const double*)E->ieps.p;
  EpiParams ep{};
  ep.inv_eps = 1.0;
  WaveTabs wt{(const double2*)E->wt_x.p, (const double2*)E->wt_y.p, (const double2*)E->wt_z.p,
              (const double2*)E->wt_pe.p, (const double2*)E->wt_ph.p, (const int*)E->wt_first.p};

  // ---- 1. admission ----
  std::vector<int> adm;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    for (int s = 0; s < S && !E->queue.empty(); ++s)
      if (E->slots[s].state == SL_FREE) {
        E->slots[s] = EngineSlot();
        E->slots[s].u = std::move(E->queue.front());
        E->queue.pop_front();
        E->slots[s].state = SL_RESIDUAL;
        E->slots[s].fresh = true;
        adm.push_back(s);
      }
  }
  if (!adm.empty()) {
    std::vector<double> ksqh(S), iepsh(S);
    FM_CK(cudaMemcpyAsync(ksqh.data(), E->ksq.p, S * sizeof(double), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaMemcpyAsync(iepsh.data(), E->ieps.p, S * sizeof(double), cudaMemcpyDeviceToHost, P->st));
    FM_CK(cudaStreamSynchronize(P->st));
    const void* last_eps = nullptr;
    double vmax = 0.0;
    const int n3[3] = {P->dims.nx, P->dims.ny, P->dims.nz};
    std::vector<double2> tx(n3[0]), ty(n3[1]), tz(n3[2]), pe(3), ph(3);
    for (int s : adm) {
      EngineSlot& sl = E->slots[s];
      // potential of the slot (the permittivity crosses once per request), as build_potential
      if (sl.u.eps_sh.get() != last_eps) {
        FM_CK(cudaMemcpyAsync(E->epsd.p, sl.u.eps_sh->data(), (size_t)g * sizeof(double2), cudaMemcpyHostToDevice,
                              P->st));
        unsigned* cnt = (unsigned*)((char*)E->maxo.p + 8);
        k_potential_max<<<592, 256, 0, P->st>>>(g, (const double2*)E->epsd.p, E->eps_bg, k2, (double*)E->maxp.p,
                                                 (double*)E->maxo.p, cnt);
        FM_CK(cudaGetLastError());
        FM_CK(cudaMemcpyAsync(&vmax, E->maxo.p, sizeof(double), cudaMemcpyDeviceToHost, P->st));
        FM_CK(cudaStreamSynchronize(P->st));
        last_eps = sl.u.eps_sh.get();
      }
      sl.eps_imag = std::max(std::pow(2.0, -20), vmax * 1.01);
      ksqh[s] = sl.eps_imag / kref2;
      iepsh[s] = kref2 / sl.eps_imag;
      k_potential_build<R><<<1184, 256, 0, P->st>>>(P->pi, (const double2*)E->epsd.p, E->eps_bg, k2, sl.eps_imag,
                                                    (const double*)P->fx.p, (const double*)P->fy.p,
                                                    (const double*)P->fz.p, 1.0 / kref2, (T*)E->Vs.p + (size_t)s * n);
      FM_CK(cudaGetLastError());
      // iteration limit of this right-hand side (convergent_born.jl:746)
      sl.maxiters = std::max(2 * engine_bornmax(P, sl.eps_imag, sl.u.itmax_setting), 100);
      FM_TRY(wave_tables(P, sl.u.src, E->eps_bg, tx.data(), ty.data(), tz.data(), pe.data(), ph.data()));
      FM_CK(cudaMemcpyAsync((double2*)E->wt_x.p + (size_t)s * n3[0], tx.data(), n3[0] * sizeof(double2),
                            cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync((double2*)E->wt_y.p + (size_t)s * n3[1], ty.data(), n3[1] * sizeof(double2),
                            cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync((double2*)E->wt_z.p + (size_t)s * n3[2], tz.data(), n3[2] * sizeof(double2),
                            cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync((double2*)E->wt_pe.p + 3 * s, pe.data(), 3 * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync((double2*)E->wt_ph.p + 3 * s, ph.data(), 3 * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaStreamSynchronize(P->st));  // host tables are reused by the next slot
    }
    FM_CK(cudaMemcpyAsync(E->ksq.p, ksqh.data(), S * sizeof(double), cudaMemcpyHostToDevice, P->st));
    FM_CK(cudaMemcpyAsync(E->ieps.p, iepsh.data(), S * sizeof(double), cudaMemcpyHostToDevice, P->st));
    for (int s = 0; s < S; ++s) acth[s] = 0;
    for (int s : adm) acth[s] = 1;
    FM_TRY(upload_act());
    k_source_term<R><<<dim3(148, S), 256, 0, P->st>>>(P->pi, S, wt, (const T*)E->Vs.p, 0.0, (T*)E->Sb.p, act,
                                                      (long long)n, (const double*)E->ksq.p);
    FM_CK(cudaGetLastError());
    // b = G S ; x = b   (warm start u0 = b)
    FM_TRY(green_op<R>(P, S, E->Sb.p, PRO_COPY, nullptr, EPI_STORE, nullptr, nullptr, ep, E->Bv.p, act,
                       (int)adm.size(), &rc));
    std::vector<cd> one(S, 1.0), zz(S);
    FM_TRY(axpby3<R>(P, S, E->Bv.p, one, nullptr, zz, nullptr, zz, E->X.p, false, act, nullptr));
  }

  // ---- 2. r0 = M^{-1}(b - A x) into U[0] for admitted and restarted slots ----
  {
    std::vector<int> res = select({SL_RESIDUAL});
    if (!res.empty()) {
      FM_TRY(upload_act());
      FM_TRY(green_op<R>(P, S, E->X.p, PRO_V, nullptr, EPI_PREC_RES, E->X.p, E->Bv.p, ep, U, act, (int)res.size(), &rc));
      std::vector<double2> hv;
      FM_TRY(multidot<R>(P, S, 0, U, U, true, act, hv, (int)res.size()));
      for (int s : res) {
        EngineSlot& sl = E->slots[s];
        sl.beta = std::sqrt(hv[s].x);
        sl.c.clear();
        sl.sn.clear();
        sl.R.clear();
        sl.z.assign(1, cd(sl.beta, 0.0));
        sl.j = 0;
        sl.inner = 0;
        if (sl.fresh) {
          sl.fresh = false;
          sl.beta0 = sl.beta;
          sl.rnorm = sl.beta;
          sl.eps = sl.u.tol * 1e-2 + sl.u.tol * sl.beta;  // abstol + reltol * ||r0||
          if (sl.beta == 0.0 || sl.rnorm <= sl.eps) {
            sl.solved = true;
            sl.state = SL_STOP;
            continue;
          }
        } else if (sl.beta == 0.0) {
          sl.solved = true;
          sl.state = SL_STOP;
          continue;
        }
        E->sch[(size_t)0 * S + s] = 1.0 / sl.beta;
        sl.state = SL_RUN;
      }
    }
  }

  // ---- 3. one GMRES iteration on every running slot ----
  {
    std::vector<int> run = select({SL_RUN});
    if (!run.empty()) {
      FM_TRY(upload_act());
      std::vector<const void*> tin(S, nullptr);
      std::vector<void*> tout(S, nullptr);
      std::vector<double> sc(S, 0.0);
      std::vector<int> kb(S, 0);
      int kmax = 0;
      for (int s : run) {
        const EngineSlot& sl = E->slots[s];
        tin[s] = U + ((size_t)sl.j * S + s) * M;
        tout[s] = U + ((size_t)(sl.j + 1) * S + s) * M;
        sc[s] = E->sch[(size_t)sl.j * S + s];
        kb[s] = sl.j + 1;
        kmax = std::max(kmax, kb[s]);
      }
      void** dt = (void**)E->tabs.p;
      FM_CK(cudaMemcpyAsync(dt, tin.data(), S * sizeof(void*), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync(dt + S, tout.data(), S * sizeof(void*), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync(E->scale.p, sc.data(), S * sizeof(double), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync(E->kb.p, kb.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
      // w = M^{-1} A v_j  (v_j = sc_j U_j) into U_{j+1}, each slot at its own j
      RhsCtx rcx = rc;
      rcx.vt.in = (const void* const*)dt;
      rcx.vt.out = (void* const*)(dt + S);
      FM_TRY(green_op<R>(P, S, U, PRO_V_SCALE, (const double*)E->scale.p, EPI_PREC_OP, U, nullptr, ep, U, act,
                         (int)run.size(), &rcx));
      // classical Gram-Schmidt (optionally twice) against each slot's own basis, FP64 coefficients
      const int nblk_d = kv_blocks(P, k_multidot<R, false>, S);
      const int nblk_u = kv_blocks(P, k_update<R, true>, S);
      const int passes = E->ortho == FM_ORTHO_CGS2 ? 2 : 1;
      std::vector<double2> htot((size_t)S * kmax, make_double2(0, 0)), hr((size_t)S * kmax);
      FM_CK(cudaMemcpyAsync(P->scale.p, E->sch.data(), (size_t)(kmax + 1) * S * sizeof(double), cudaMemcpyHostToDevice,
                            P->st));
      for (int pass = 0; pass < passes; ++pass) {
        const double fbA = (double)run.size() * M * sizeof(T);
        FM_TRACK(P, KC_DOT, (kmax + 1) * fbA,
                 (k_multidot<R, false><<<dim3(nblk_d, S), KV_THREADS, 0, P->st>>>(
                     P->M, S, kmax, U, nullptr, (double2*)P->red_part.p, (double2*)P->red_out.p,
                     (unsigned*)P->red_cnt.p, act, (const T* const*)(dt + S), (const int*)E->kb.p)));
        FM_CK(cudaGetLastError());
        FM_CK(cudaMemcpyAsync(hr.data(), P->red_out.p, hr.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
        FM_CK(cudaStreamSynchronize(P->st));
        for (int s : run)
          for (int i = 0; i < kb[s]; ++i) {
            const double sci = E->sch[(size_t)i * S + s];
            htot[(size_t)s * kmax + i].x += hr[(size_t)s * kmax + i].x * sci;
            htot[(size_t)s * kmax + i].y += hr[(size_t)s * kmax + i].y * sci;
          }
        FM_CK(cudaMemcpyAsync(P->coef.p, hr.data(), hr.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
        Coef cf{(const double2*)P->coef.p, kmax, (const double*)P->scale.p, S, -1.0, 0};
        FM_TRACK(P, KC_UPD, (kmax + 2) * fbA,
                 (k_update<R, true><<<dim3(nblk_u, S), KV_THREADS, 0, P->st>>>(
                     P->M, S, kmax, U, cf, nullptr, nullptr, (double2*)P->red_part.p, (double2*)P->red_out.p,
                     (unsigned*)P->red_cnt.p, act, (T* const*)(dt + S), (const int*)E->kb.p)));
        FM_CK(cudaGetLastError());
      }
      std::vector<double2> nn(S);
      FM_CK(cudaMemcpyAsync(nn.data(), P->red_out.p, S * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
      FM_CK(cudaStreamSynchronize(P->st));
      tk_resolve(P);
      // Givens update per slot (Krylov.jl gmres)
      for (int s : run) {
        EngineSlot& sl = E->slots[s];
        const int K = sl.j + 1;
        std::vector<cd> col(K);
        for (int i = 0; i < K; ++i) col[i] = cd(htot[(size_t)s * kmax + i].x, htot[(size_t)s * kmax + i].y);
        const double hb = std::sqrt(std::max(0.0, nn[s].x));
        for (int i = 0; i < K - 1; ++i) {
          cd t = sl.c[i] * col[i] + sl.sn[i] * col[i + 1];
          col[i + 1] = std::conj(sl.sn[i]) * col[i] - sl.c[i] * col[i + 1];
          col[i] = t;
        }
        double c;
        cd sn, rho;
        sym_givens(col[K - 1], hb, c, sn, rho);
        col[K - 1] = rho;
        sl.c.push_back(c);
        sl.sn.push_back(sn);
        sl.R.push_back(col);
        const cd zk1 = std::conj(sn) * sl.z[K - 1];
        sl.z[K - 1] = c * sl.z[K - 1];
        sl.rnorm = std::abs(zk1);
        sl.inner = K;
        sl.iters += 1;
        const bool solved = sl.rnorm <= sl.eps || sl.rnorm + 1.0 <= 1.0;
        sl.solved = solved;
        if (solved || hb <= btol || sl.iters >= sl.maxiters) {
          sl.state = SL_STOP;
        } else if (K >= E->mem) {
          sl.state = SL_RESTART;
        } else {
          sl.z.push_back(zk1);
          E->sch[(size_t)(sl.j + 1) * S + s] = 1.0 / hb;
          sl.j += 1;
        }
      }
    }
  }

  // ---- 4. x += sum_i y_i v_i for slots whose cycle ended ----
  {
    std::vector<int> upd = select({SL_STOP, SL_RESTART});
    std::vector<double2> yh((size_t)S * (KV_KMAX + 1), make_double2(0, 0));
    std::vector<int> kb(S, 0);
    int kmax = 0;
    for (int s : upd) {
      EngineSlot& sl = E->slots[s];
      const int n_in = sl.inner;
      if (n_in == 0) continue;
      std::vector<cd> y(sl.z.begin(), sl.z.begin() + n_in);
      for (int i = n_in - 1; i >= 0; --i) {
        for (int jj = n_in - 1; jj > i; --jj) y[i] -= sl.R[jj][i] * y[jj];
        if (std::abs(sl.R[i][i]) <= btol) {
          for (int q = 0; q <= i; ++q) y[q] = 0.0;
          break;
        }
        y[i] /= sl.R[i][i];
      }
      for (int i = 0; i < n_in; ++i) yh[(size_t)s * (KV_KMAX + 1) + i] = make_double2(y[i].real(), y[i].imag());
      kb[s] = n_in;
      kmax = std::max(kmax, n_in);
      sl.inner = 0;
    }
    if (kmax > 0) {
      FM_TRY(upload_act());
      FM_CK(cudaMemcpyAsync(E->kb.p, kb.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync(P->coef.p, yh.data(), yh.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_CK(cudaMemcpyAsync(P->scale.p, E->sch.data(), (size_t)(kmax + 1) * S * sizeof(double), cudaMemcpyHostToDevice,
                            P->st));
      Coef cf{(const double2*)P->coef.p, KV_KMAX + 1, (const double*)P->scale.p, S, 1.0, 1};
      FM_TRACK(P, KC_UPD, (double)(kmax + 2) * upd.size() * M * sizeof(T),
               (k_update<R, false><<<dim3(kv_blocks(P, k_update<R, false>, S), S), KV_THREADS, 0, P->st>>>(
                   P->M, S, kmax, U, cf, (T*)E->X.p, nullptr, nullptr, nullptr, nullptr, act, nullptr,
                   (const int*)E->kb.p)));
      FM_CK(cudaGetLastError());
    }
    for (int s : upd)
      if (E->slots[s].state == SL_RESTART) E->slots[s].state = SL_RESIDUAL;
  }

  // ---- 5. finish the slots that stopped ----
  {
    std::vector<int> fin = select({SL_STOP});
    if (!fin.empty()) {
      FM_TRY(upload_act());
      FM_TRY(curl_batch<R>(P, S, E->X.p, E->Hb.p, act));
      k_assemble<R><<<dim3(148, S), 256, 0, P->st>>>(P->pi, S, wt, (const T*)E->X.p, (const T*)E->Hb.p,
                                                     (double2*)E->Eo.p, (double2*)E->Ho.p, act);
      FM_CK(cudaGetLastError());
      for (int s : fin) {
        EngineSlot& sl = E->slots[s];
        FM_CK(cudaMemcpyAsync(sl.u.E_out, (double2*)E->Eo.p + (size_t)s * 3 * g, 3 * g * sizeof(double2),
                              cudaMemcpyDeviceToHost, P->st));
        FM_CK(cudaMemcpyAsync(sl.u.H_out, (double2*)E->Ho.p + (size_t)s * 3 * g, 3 * g * sizeof(double2),
                              cudaMemcpyDeviceToHost, P->st));
      }
      FM_CK(cudaStreamSynchronize(P->st));
      tk_resolve(P);
      FM_TRY(check_device_error(P));
      std::lock_guard<std::mutex> lk(E->mu);
      for (int s : fin) {
        EngineSlot& sl = E->slots[s];
        fm_solve_info inf{};
        inf.iterations = sl.iters;
        inf.solved = sl.solved ? 1 : 0;
        inf.residual = sl.rnorm;
        inf.residual0 = sl.beta0;
        E->done.push_back({sl.u.req, sl.u.rhs, inf});
        sl = EngineSlot();
      }
    }
  }
  return FM_OK;
}

fm_status fm_engine_step(fm_engine* E, int* n_done, long long* done_req, int* done_rhs, fm_solve_info* done_info,
                         int max_done) {
  if (!E) return fail(FM_ERR_INVALID, "null engine");
  FM_CK(cudaSetDevice(E->P->desc.device));
  fm_status st = E->P->prec == FM_PREC_F64 ? engine_step_t<double>(E) : engine_step_t<float>(E);
  if (st != FM_OK) return st;
  std::lock_guard<std::mutex> lk(E->mu);
  int k = 0;
  while (k < max_done && !E->done.empty()) {
    const auto d = E->done.front();
    E->done.pop_front();
    if (done_req) done_req[k] = d.req;
    if (done_rhs) done_rhs[k] = d.rhs;
    if (done_info) done_info[k] = d.info;
    ++k;
  }
  if (n_done) *n_done = k;
  return FM_OK;
}
