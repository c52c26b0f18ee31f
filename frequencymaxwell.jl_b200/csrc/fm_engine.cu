// libfmcuda: the slot engine behind the serving loop (continuous batching of independent right-hand sides).
#include "fm_plan.cuh"
#include "fm_blockalg.h"

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
//
// With FM_ORTHO_BLOCK every slot runs s-step block GMRES (s = 8, FP64 block
// vectors stored orthonormalised, the per-RHS algebra of the batched block solve,
// fm_blockalg.cu): the first s iterations of a cycle share step 3's CGS launches,
// after which each engine step advances the slot by one block of s iterations
// (3b), in launches shared by every slot in that phase, each at its own basis
// size.  A slot whose limit fits the basis (maxiters + s + 1 stored vectors) runs
// full GMRES as the batched block solve does; otherwise it restarts when the
// basis is full, every floor(basis / s) * s iterations (s-step GMRES(m), the
// restart points of CGS GMRES(basis) when s divides the basis).
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
  bool blk = false;    // s-step block GMRES (FM_ORTHO_BLOCK engines, limit fits the basis)
  int phase = 0;       // block slots: 1 = the first s CGS steps of a cycle, 2 = blocks
  int m = 0;           // block slots: Hessenberg columns done in this cycle
  int itbase = 0;      // block slots: iterations of the cycles before this one
  BlkState bst;
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
  int bs = 0;  // FM_ORTHO_BLOCK: vectors per block
  DevBuf U, X, Bv, Sb, Hb, Vs, ksq, ieps, scale, act, kb, tabs, Eo, Ho, wt_x, wt_y, wt_z, wt_pe, wt_ph, wt_first,
      epsd, maxp, maxo;
  DevBuf Yb, V64s, k0d, ncd, vrowd, kbd;  // block slots: FP64 block vectors, FP64 potentials, per-slot indices
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

// vectors per block of the engine's block GMRES
static constexpr int kEngineBlock = 8;

long long fm_engine_slot_bytes_ortho(const fm_plan_desc* d, int basis, int ortho) {
  const long long base = fm_engine_slot_bytes(d, basis);
  if (base < 0 || ortho != FM_ORTHO_BLOCK) return base;
  long long n = 1;
  for (int a = 0; a < 3; ++a) n *= (long long)(d->grid[a] + 2 * d->pad[a]);
  const long long esz = d->precision == FM_PREC_F64 ? 16 : 8, ysz = d->precision == FM_PREC_F32 ? 8 : 16;
  // block vectors Y_0..Y_s, the pass temporaries at the block-vector type, a potential of that type
  return base + 3 * n * ysz * (kEngineBlock + 1) + 2 * 3 * n * (ysz - esz) + (ysz != esz ? n * ysz : 0);
}

fm_status fm_engine_create(fm_plan* P, int slots, int basis, double wavelength, double eps_bg, const double* fx,
                           const double* fy, const double* fz, int ortho, fm_engine** out) {
  if (!P || !out || slots < 1 || basis < 1) return fail(FM_ERR_INVALID, "fm_engine_create: bad argument");
  *out = nullptr;
  if (basis + 1 > KV_KMAX) return fail(FM_ERR_UNSUPPORTED, "Krylov basis larger than 127 vectors");
  if (!(wavelength > 0) || !(eps_bg > 0)) return fail(FM_ERR_INVALID, "wavelength and permittivity_bg must be positive");
  if (ortho != FM_ORTHO_CGS && ortho != FM_ORTHO_CGS2 && ortho != FM_ORTHO_BLOCK)
    return fail(FM_ERR_INVALID, "the engine runs CGS, CGS2 or block GMRES");
  FM_CK(cudaSetDevice(P->desc.device));
  fm_engine* E = new fm_engine();
  E->P = P;
  E->S = slots;
  E->mem = basis;
  E->ortho = ortho;
  E->bs = ortho == FM_ORTHO_BLOCK ? kEngineBlock : 0;
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
  // block slots: block vectors, pass temporaries and potentials of the block-vector type (FP64 unless the plan
  // computes in FP32), per-slot index arrays, update coefficients of a whole block
  const size_t ysz = P->c64 ? sizeof(double2) : esz, tsz = E->bs ? std::max(esz, ysz) : esz;
  if (E->bs) {
    al(E->Yb, (size_t)(E->bs + 1) * S * M * ysz);
    if (ysz != esz) al(E->V64s, S * n * ysz);
    al(E->k0d, S * sizeof(int));
    al(E->ncd, S * sizeof(int));
    al(E->vrowd, S * sizeof(int));
    al(E->kbd, S * sizeof(int));
    if (e == cudaSuccess) e = P->shifts.ensure(S * sizeof(double2));
  }
  if (e == cudaSuccess) e = P->t1.ensure(S * M * tsz);
  if (e == cudaSuccess) e = P->t2.ensure(S * M * tsz);
  if (e == cudaSuccess) e = P->scale.ensure((size_t)(KV_KMAX + 1) * S * sizeof(double));
  if (e == cudaSuccess)
    e = P->coef.ensure((size_t)(KV_KMAX + 1) * S * std::max(E->bs, 1) * sizeof(double2));
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
  DevBuf* b[] = {&E->U,    &E->X,    &E->Bv,    &E->Sb,       &E->Hb,   &E->Vs,   &E->ksq,  &E->ieps,
                 &E->scale, &E->act,  &E->kb,    &E->tabs,     &E->Eo,   &E->Ho,   &E->wt_x, &E->wt_y,
                 &E->wt_z,  &E->wt_pe, &E->wt_ph, &E->wt_first, &E->epsd, &E->maxp, &E->maxo, &E->Yb,
                 &E->V64s,  &E->k0d,  &E->ncd,   &E->vrowd,    &E->kbd};
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

// One s-step block (fm_blockalg.cu) on every running block slot in its second phase, each at its own column m
// (basis size m + 1): start vectors, s shifted operator applications on the FP64 block vectors, the block dot,
// the in-place update and its Gram matrix, and the orthonormalised block stored after each slot's basis.
template <typename R, typename YR>
static fm_status engine_block_step(fm_engine* E, std::vector<int>& acth, const RhsCtx& rc) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  fm_plan* P = E->P;
  const int S = E->S, bs = E->bs;
  const size_t fe = (size_t)P->M;
  std::vector<int> run;
  for (int s = 0; s < S; ++s) {
    const EngineSlot& sl = E->slots[s];
    acth[s] = sl.state == SL_RUN && sl.blk && sl.phase == 2;
    if (acth[s]) run.push_back(s);
  }
  if (run.empty()) return FM_OK;
  const int nact = (int)run.size();
  int* act = (int*)E->act.p;
  T* U = (T*)E->U.p;
  TY* Yb = (TY*)E->Yb.p;
  FM_CK(cudaMemcpyAsync(act, acth.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
  // Y_0 = V_m of each slot (a combination of the stored vectors of m's diagonal block)
  int Kmax = 0;
  std::vector<int> kh(S, 0), k0h(S, 0), nch(S, 0);
  std::vector<double2> cc((size_t)S * 16, make_double2(0, 0));
  for (int s : run) {
    const EngineSlot& sl = E->slots[s];
    kh[s] = sl.m + 1;
    k0h[s] = blk_start(sl.bst, sl.m, cc.data() + (size_t)s * 16);
    nch[s] = sl.m - k0h[s] + 1;
    Kmax = std::max(Kmax, kh[s]);
  }
  FM_CK(cudaMemcpyAsync(E->kbd.p, kh.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
  FM_CK(cudaMemcpyAsync(E->vrowd.p, kh.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
  FM_CK(cudaMemcpyAsync(E->k0d.p, k0h.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
  FM_CK(cudaMemcpyAsync(E->ncd.p, nch.data(), S * sizeof(int), cudaMemcpyHostToDevice, P->st));
  FM_CK(cudaMemcpyAsync(P->coef.p, cc.data(), cc.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
  double ncs = 0;
  for (int s : run) ncs += nch[s];
  FM_TRACK(P, KC_AXPBY, (ncs * sizeof(T) + nact * sizeof(TY)) * (double)fe,
           (k_combine<R, TY><<<dim3(2 * P->sms, S), KV_THREADS, 0, P->st>>>(
               P->M, S, 0, 1, U, (const double2*)P->coef.p, 16, Yb, act, (const int*)E->k0d.p,
               (const int*)E->ncd.p)));
  FM_CK(cudaGetLastError());
  // Y_t = M^{-1}A Y_{t-1} - theta_t Y_{t-1}, t = 1..s, with each slot's potential and shifts
  RhsCtx rcY = rc;
  rcY.V = sizeof(TY) != sizeof(T) ? E->V64s.p : E->Vs.p;
  EpiParams ep{};
  ep.inv_eps = 1.0;
  std::vector<double2> th(S, make_double2(0, 0));
  for (int t = 1; t <= bs; ++t) {
    for (int s : run)
      th[s] = make_double2(E->slots[s].bst.theta[t - 1].real(), E->slots[s].bst.theta[t - 1].imag());
    FM_CK(cudaMemcpyAsync(P->shifts.p, th.data(), S * sizeof(double2), cudaMemcpyHostToDevice, P->st));
    EpiParams eps = ep;
    eps.shift_b = (const double2*)P->shifts.p;
    TY* Yin = Yb + (size_t)(t - 1) * S * fe;
    TY* Yout = Yb + (size_t)t * S * fe;
    FM_TRY(green_op<YR>(P, S, Yin, PRO_V, nullptr, EPI_PREC_OP, Yin, nullptr, eps, Yout, act, nact, &rcY));
  }
  // D = X^H Y_{1..s} (rows past each slot's basis come out zero)
  const int* kbd = (const int*)E->kbd.p;
  FM_CK((block_kernels<R, YR>(P, 0, bs, S, Kmax, U, Yb + (size_t)S * fe, nullptr, act, nact, kbd)));
  std::vector<double2> D((size_t)S * Kmax * bs);
  FM_CK(cudaMemcpyAsync(D.data(), P->red_out.p, D.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  tk_resolve(P);
  std::vector<std::vector<cd>> Cv(S);
  std::vector<double2> cf((size_t)S * KV_KMAX * bs, make_double2(0, 0));
  for (int s : run)
    blk_project(E->slots[s].bst, E->slots[s].m, bs, D.data() + (size_t)s * Kmax * bs, Cv[s],
                cf.data() + (size_t)s * KV_KMAX * bs);
  FM_CK(cudaMemcpyAsync(P->coef.p, cf.data(), cf.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
  // Y' = Y - X E in place, and its Gram matrix
  FM_CK((block_kernels<R, YR>(P, 2, bs, S, Kmax, U, Yb + (size_t)S * fe, Yb + (size_t)S * fe, act, nact, kbd)));
  const int NG = bs <= 8 ? bs * (bs + 1) / 2 : bs * bs;
  std::vector<double2> Gt((size_t)S * NG);
  FM_CK(cudaMemcpyAsync(Gt.data(), P->red_out.p, Gt.size() * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  tk_resolve(P);
  std::vector<double2> rbi((size_t)S * bs * bs, make_double2(0, 0));
  for (int s : run) {
    EngineSlot& sl = E->slots[s];
    const bool stop = blk_absorb(sl.bst, sl.m, bs, true, Gt.data() + (size_t)s * NG, Cv[s],
                                 rbi.data() + (size_t)s * bs * bs, sl.maxiters - sl.itbase);
    sl.iters = sl.itbase + sl.bst.iters;
    sl.rnorm = sl.bst.rnorm;
    sl.solved = sl.bst.solved;
    if (stop) {
      sl.state = SL_STOP;
    } else {
      sl.m += bs;
      if (sl.m + bs > E->mem) sl.state = SL_RESTART;  // the next block would not fit: end the cycle
    }
  }
  // V = Y' Rb^{-1} into each slot's basis rows m+1 .. m+s (also for slots that stopped in this block: their
  // solution uses these vectors; a block that lost rank gets zero coefficients and is not used)
  FM_CK(cudaMemcpyAsync(P->coef.p, rbi.data(), rbi.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
  FM_CK((block_kernels<R, YR>(P, 3, bs, S, 0, U, Yb + (size_t)S * fe, U, act, nact, (const int*)E->vrowd.p)));
  return FM_OK;
}

template <typename R, typename YR>
static fm_status engine_step_t(fm_engine* E) {
  using T = cplx<R>;
  using TY = cplx<YR>;
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
      const bool v64 = E->bs && sizeof(TY) != sizeof(T);
      if (E->Vs.cap < (size_t)(s + 1) * n * sizeof(T) || (v64 && E->V64s.cap < (size_t)(s + 1) * n * sizeof(double2)))
        return fail(FM_ERR_INVALID, "engine potential buffers smaller than the slots");
      k_potential_build<R><<<1184, 256, 0, P->st>>>(P->pi, (const double2*)E->epsd.p, E->eps_bg, k2, sl.eps_imag,
                                                    (const double*)P->fx.p, (const double*)P->fy.p,
                                                    (const double*)P->fz.p, 1.0 / kref2, (T*)E->Vs.p + (size_t)s * n);
      FM_CK(cudaGetLastError());
      if (v64) {  // the block vectors' operator reads the same potential widened to FP64
        k_to_f64<R><<<2 * P->sms, 256, 0, P->st>>>((long long)n, (const T*)E->Vs.p + (size_t)s * n, 1.0,
                                                   (double2*)E->V64s.p + (size_t)s * n);
        FM_CK(cudaGetLastError());
      }
      // iteration limit of this right-hand side (convergent_born.jl:746)
      sl.maxiters = std::max(2 * engine_bornmax(P, sl.eps_imag, sl.u.itmax_setting), 100);
      sl.blk = E->bs > 0 && E->mem >= 2 * E->bs && (M & 3) == 0;
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
          if (sl.blk) {
            sl.m = sl.j = 0;
            sl.phase = 1;
            sl.itbase = 0;
            if (blk_init(sl.bst, E->mem + 2, sl.beta, sl.u.tol * 1e-2, sl.u.tol)) {
              sl.solved = true;
              sl.state = SL_STOP;
              continue;
            }
          } else if (sl.beta == 0.0 || sl.rnorm <= sl.eps) {
            sl.solved = true;
            sl.state = SL_STOP;
            continue;
          }
        } else if (sl.beta == 0.0) {
          sl.solved = true;
          sl.state = SL_STOP;
          continue;
        } else if (sl.blk) {  // the next cycle of a block slot: a new basis from the updated residual
          sl.itbase = sl.iters;
          blk_restart(sl.bst, E->mem + 2, sl.beta, sl.eps);
          sl.m = sl.j = 0;
          sl.phase = 1;
        }
        E->sch[(size_t)0 * S + s] = 1.0 / sl.beta;
        sl.state = SL_RUN;
      }
    }
  }

  // ---- 3. one GMRES iteration on every running slot (block slots: their first s steps) ----
  {
    std::vector<int> run = select({SL_RUN});
    for (size_t q = 0; q < run.size();) {
      const EngineSlot& sl = E->slots[run[q]];
      if (sl.blk && sl.phase == 2) {
        acth[run[q]] = 0;
        run.erase(run.begin() + q);
      } else {
        ++q;
      }
    }
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
        if (sl.blk) {  // Hessenberg column m of the block solve, its Givens update and stop test
          BlkState& r = sl.bst;
          for (int i = 0; i < K; ++i) r.H[i + (size_t)sl.m * r.ld] = col[i];
          const bool stop = blk_cgs_close(r, sl.m, hb, sl.maxiters - sl.itbase);
          sl.iters = sl.itbase + r.iters;
          sl.rnorm = r.rnorm;
          sl.solved = r.solved;
          if (stop) {
            sl.state = SL_STOP;
            continue;
          }
          E->sch[(size_t)(sl.m + 1) * S + s] = 1.0 / hb;
          sl.j = ++sl.m;
          if (sl.m == E->bs) {  // Newton shifts: Ritz values of the leading s x s Hessenberg block, Leja ordered
            r.theta.assign(E->bs, 0.0);
            blk_shifts(r, 0, E->bs);
            sl.phase = 2;
          }
          continue;
        }
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

  // ---- 3b. one s-step block on every block slot past its first s steps ----
  if (E->bs) FM_TRY((engine_block_step<R, YR>(E, acth, rc)));

  // ---- 4. x += sum_i y_i v_i for slots whose cycle ended ----
  {
    std::vector<int> upd = select({SL_STOP, SL_RESTART});
    std::vector<double2> yh((size_t)S * (KV_KMAX + 1), make_double2(0, 0));
    std::vector<int> kb(S, 0);
    int kmax = 0;
    for (int s : upd) {
      EngineSlot& sl = E->slots[s];
      if (sl.blk) {  // X coordinates: the stored vectors enter unscaled
        const int nv = blk_solution(sl.bst, yh.data() + (size_t)s * (KV_KMAX + 1));
        for (int i = 0; i < nv; ++i) E->sch[(size_t)i * S + s] = 1.0;
        kb[s] = nv;
        kmax = std::max(kmax, nv);
        continue;
      }
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
  fm_status st = E->P->prec == FM_PREC_F64 ? engine_step_t<double, double>(E)
                 : E->P->c64              ? engine_step_t<float, double>(E)
                                          : engine_step_t<float, float>(E);
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

