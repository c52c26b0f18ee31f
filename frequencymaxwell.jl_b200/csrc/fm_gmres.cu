// libfmcuda: the Krylov drivers of the CBS solve -- GMRES (Krylov.jl semantics: MGS / CGS / CGS2, GMRES(m)),
// s-step block GMRES on the FP64 tensor cores, BiCGStab and the plain Born series -- and the solve core that
// runs them from source terms to the scattered field and its curl.
#include "fm_plan.cuh"
#include "fm_blockalg.h"

// ---------------------------------------------------------------------------
// Krylov helpers
// ---------------------------------------------------------------------------
template <typename R>
fm_status multidot(fm_plan* P, int nb, int K, const void* U, const void* w, bool wnorm, const int* act,
                   std::vector<double2>& host_out, int nact) {
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
fm_status axpby3(fm_plan* P, int nb, const void* a, const std::vector<cd>& ca, const void* b,
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

void sym_givens(cd a, double b, double& c, cd& s, cd& rho) {
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

double now_s() {
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
// The per-RHS algebra (state, triangular solves, Hessenberg recovery, shifts, Givens) is in fm_blockalg.cu.


template <typename R, typename YR, int S>
static cudaError_t launch_blockdot(fm_plan* P, int nb, int K, const void* U, const void* Y, const int* act, int nact,
                                   const int* Kb) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  const double bytes = ((double)K * sizeof(T) + (double)S * sizeof(TY)) * nact * P->M;
  const size_t pb =
      P->bd_bulk ? blockdot_bulk_part_bytes((int)sizeof(R), (int)sizeof(YR), S, P->M, nb, nact, K, P->sms) : 0;
  if (pb && !Kb) {
    cudaError_t e = P->red_part.ensure(pb);
    if (e == cudaSuccess) e = P->red_out.ensure((size_t)nb * (std::max)(K * S, KV_KMAX + 2) * sizeof(double2));
    if (e != cudaSuccess) return e;
    FM_TRACK(P, KC_DOT, bytes,
             e = launch_blockdot_bulk((int)sizeof(R), (int)sizeof(YR), S, P->M, nb, nact, K, U, Y,
                                      (double2*)P->red_part.p, P->red_part.cap, (double2*)P->red_out.p,
                                      (unsigned*)P->red_cnt.p, act, (int*)P->errbuf.p, P->sms, P->st));
    return e;
  }
  // register kernel: two groups of 8 basis vectors per warp (tuning 0) or four (tuning 2, 5 <= S <= 8)
  const bool wide = P->bd_wide && S > 4 && S <= 8;
  auto kern = wide ? k_blockdot_mma<R, TY, S, (S > 4 && S <= 8)> : k_blockdot_mma<R, TY, S, false>;
  // CTA shape: KW warps along the basis times EW along the elements, with KW * EW <= KV_WARPS and no idle warp
  // (a basis of 9..16 groups of 8 vectors would otherwise leave up to 3 of 8 warps without work)
  const int KG = (K + 7) / 8, GPW = (S <= 4 || wide) ? 4 : 2, KW = (KG + GPW - 1) / GPW;
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
                                                         (unsigned*)P->red_cnt.p, act, Kb)));
  return cudaGetLastError();
}

// Z = Y - X E and the Gram matrix of Z.  TZ: type of Z (the basis type, or the block-vector type when the block
// is stored orthonormalised afterwards and Z overwrites Y in place).  The Gram goes to red_out: the upper triangle
// tri(t,u) for S <= 8 (accumulated by the update kernel itself from the values it stores), the full S x S matrix
// <Z_t, Z_u> at t*S + u for S > 8 (the block dot of Z against itself on the tensor cores, a second pass).
template <typename R, typename YR, int S, typename TZ>
static cudaError_t launch_blockupdate(fm_plan* P, int nb, int K, const void* U, const void* Y, void* Z, const int* act,
                                      int nact, const int* Kb) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  constexpr int NG = S * (S + 1) / 2;
  constexpr int TILE = S <= 8 ? 32 : 16;  // elements per warp tile of k_blockupdate_mma
  auto kern = k_blockupdate_mma<R, TY, S, TZ, (S <= 8)>;
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, KV_THREADS, 0) != cudaSuccess || bps < 1) bps = 1;
  const long long maxb = (P->M + TILE * KV_WARPS - 1) / (TILE * KV_WARPS);
  const int nblk = (int)std::max(1LL, std::min<long long>(maxb, (long long)P->sms * bps / nb));
  cudaError_t e = cudaSuccess;
  if constexpr (S <= 8) {
    e = P->red_part.ensure((size_t)nb * nblk * NG * sizeof(double2));
    if (e == cudaSuccess) e = P->red_out.ensure((size_t)nb * (std::max)(NG, KV_KMAX + 2) * sizeof(double2));
    if (e != cudaSuccess) return e;
  }
  FM_TRACK(P, KC_UPD, ((double)K * sizeof(T) + (double)S * (sizeof(TY) + sizeof(TZ))) * nact * P->M,
           (kern<<<dim3(nblk, nb), KV_THREADS, 0, P->st>>>(P->M, nb, K, (const T*)U, (const TY*)Y, (TZ*)Z,
                                                            (const double2*)P->coef.p, act, Kb,
                                                            (double2*)P->red_part.p, (double2*)P->red_out.p,
                                                            (unsigned*)P->red_cnt.p)));
  e = cudaGetLastError();
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
                                                             (unsigned*)P->red_cnt.p, act, nullptr)));
    return cudaGetLastError();
  }
  return cudaSuccess;
}

// V (basis slots) = Z Rb^{-1} for the orthonormalised block storage; coefficients in P->coef
template <typename R, typename YR, int S>
static cudaError_t launch_blocknorm(fm_plan* P, int nb, const void* Z, void* V, const int* act, int nact,
                                    const int* vrow) {
  using T = cplx<R>;
  using TY = cplx<YR>;
  FM_TRACK(P, KC_AXPBY, (double)S * (sizeof(TY) + sizeof(T)) * nact * P->M,
           (k_blocknorm<R, TY, S><<<dim3(kv_blocks(P, k_blocknorm<R, TY, S>, nb), nb), KV_THREADS, 0, P->st>>>(
               P->M, nb, (const TY*)Z, (const double2*)P->coef.p, (T*)V, act, vrow)));
  return cudaGetLastError();
}

// (declared in fm_plan.cuh)
template <typename R, typename YR>
cudaError_t block_kernels(fm_plan* P, int which, int S, int nb, int K, const void* U, const void* Y, void* Z,
                          const int* act, int nact, const int* Kb) {
  using T = cplx<R>;
  using TY = cplx<YR>;
#define FM_BLK(SS)                                                                                     \
  case SS:                                                                                             \
    return which == 0   ? launch_blockdot<R, YR, SS>(P, nb, K, U, Y, act, nact, Kb)                    \
           : which == 1 ? launch_blockupdate<R, YR, SS, T>(P, nb, K, U, Y, Z, act, nact, Kb)          \
           : which == 2 ? launch_blockupdate<R, YR, SS, TY>(P, nb, K, U, Y, Z, act, nact, Kb)         \
                        : launch_blocknorm<R, YR, SS>(P, nb, Y, Z, act, nact, Kb);
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

  // r0 = M^{-1}(b - A x) into X_0
  FM_TRY(upload_active());
  FM_TRY(green_op<R>(P, nb, P->xbuf.p, PRO_V, nullptr, EPI_PREC_RES, P->xbuf.p, P->bbuf.p, ep, U, act));
  std::vector<double2> hv;
  FM_TRY(multidot<R>(P, nb, 0, U, U, true, act, hv));
  for (int b = 0; b < nb; ++b) {
    if (blk_init(St[b], ld, std::sqrt(hv[b].x), o.abstol, o.reltol)) acth[b] = 0;
    info[b].residual0 = St[b].beta;
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
    for (int b = 0; b < nb; ++b)
      if (acth[b]) blk_cgs_coefs(St[b], m, hr.data() + (size_t)b * K, cf.data() + (size_t)b * K);
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
    for (int b = 0; b < nb; ++b)
      if (acth[b] && blk_cgs_close(St[b], m, std::sqrt(std::max(0.0, nn[b].x)), itmax)) {
        St[b].active = false;
        acth[b] = 0;
      }
    ++m;
    if (deadline > 0 && now_s() > deadline) return fail(FM_ERR_TIMEOUT, "solve deadline passed");
  }
  // Newton shifts: Ritz values of the leading S x S Hessenberg block, Leja ordered
  for (int b = 0; b < nb; ++b) {
    St[b].theta.assign(S, 0.0);
    if (St[b].active) blk_shifts(St[b], 0, S);
  }

  // ---- phase 2: s-step blocks ----
  while (count_active() > 0 && m < itmax) {
    const int nact = count_active();
    FM_TRY(upload_active());
    const int K = m + 1;
    // Y_0 = V_m = sum_k X_k (Rf^{-1})_{k,m} over m's diagonal block (the same block layout for every RHS)
    int k0 = m;
    {
      std::vector<double2> cc((size_t)nb * 16, make_double2(0, 0));
      for (int b = 0; b < nb; ++b)
        if (acth[b]) k0 = blk_start(St[b], m, cc.data() + (size_t)b * 16);
      const int nc = m - k0 + 1;
      FM_CK(cudaMemcpyAsync(P->coef.p, cc.data(), cc.size() * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      FM_TRACK(P, KC_AXPBY, (double)nc * nact * fe * sizeof(T) + (double)nact * fe * sizeof(TY),
               (k_combine<R, TY><<<dim3(2 * P->sms, nb), KV_THREADS, 0, P->st>>>(
                   P->M, nb, k0, nc, U, (const double2*)P->coef.p, 16, Yb, act)));
      FM_CK(cudaGetLastError());
    }
    // Y_t = M^{-1}A Y_{t-1} - theta_t Y_{t-1}, t = 1..S; on the fused passes the x pass of application t+1 runs
    // inside the last pass of application t (GREEN_CHAIN_*), so Y_t and V are not read back for it
    const bool chainable = green_chain_ok(P, &rcY);
    std::vector<double2> th(nb);
    for (int t = 1; t <= S; ++t) {
      for (int b = 0; b < nb; ++b) th[b] = make_double2(St[b].theta[t - 1].real(), St[b].theta[t - 1].imag());
      FM_CK(cudaMemcpyAsync(P->shifts.p, th.data(), nb * sizeof(double2), cudaMemcpyHostToDevice, P->st));
      EpiParams eps = ep;
      eps.shift_b = (const double2*)P->shifts.p;
      TY* Yin = Yb + (size_t)(t - 1) * nb * fe;
      TY* Yout = Yb + (size_t)t * nb * fe;
      // (the shift array is rewritten for the next vector in stream order, after this pass has read it)
      const int chain = !chainable ? 0 : (t > 1 ? GREEN_CHAIN_HAVE_XF : 0) | (t < S ? GREEN_CHAIN_NEXT_XF : 0);
      FM_TRY(green_op<YR>(P, nb, Yin, PRO_V, nullptr, EPI_PREC_OP, Yin, nullptr, eps, Yout, act, nact, &rcY, chain));
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
    for (int b = 0; b < nb; ++b)
      if (acth[b]) blk_project(St[b], m, S, D.data() + (size_t)b * K * S, Cv[b], cf.data() + (size_t)b * KV_KMAX * S);
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
    for (int b = 0; b < nb; ++b)
      if (acth[b] && blk_absorb(St[b], m, S, ortho_store, Gt.data() + (size_t)b * NG, Cv[b],
                                ortho_store ? rbi.data() + (size_t)b * S * S : nullptr, itmax))
        acth[b] = 0;
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
  for (int b = 0; b < nb; ++b) Kmax = std::max(Kmax, blk_solution(St[b], yh.data() + (size_t)b * KV_KMAX));
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
fm_status check_device_error(fm_plan* P) {
  int code = 0;
  FM_CK(cudaMemcpyAsync(&code, P->errbuf.p, sizeof(int), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  if (code) {
    cudaMemsetAsync(P->errbuf.p, 0, sizeof(int), P->st);
    return fail(FM_ERR_TIMEOUT, "a TMA pipeline wait timed out on the device (code " + std::to_string(code) + ")");
  }
  return FM_OK;
}

// ---------------------------------------------------------------------------
// shared solve core: from scaled source terms in P->sbuf (nb RHS) to the
// scattered field in P->xbuf and its curl in P->ebuf.
template <typename R>
fm_status solve_core(fm_plan* P, int nb, const fm_solve_opts& o, std::vector<fm_solve_info>& info) {
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

template fm_status multidot<float>(fm_plan*, int, int, const void*, const void*, bool, const int*,
                                   std::vector<double2>&, int);
template fm_status multidot<double>(fm_plan*, int, int, const void*, const void*, bool, const int*,
                                    std::vector<double2>&, int);
template fm_status axpby3<float>(fm_plan*, int, const void*, const std::vector<cd>&, const void*,
                                 const std::vector<cd>&, const void*, const std::vector<cd>&, void*, bool,
                                 const int*, std::vector<double>*);
template fm_status axpby3<double>(fm_plan*, int, const void*, const std::vector<cd>&, const void*,
                                  const std::vector<cd>&, const void*, const std::vector<cd>&, void*, bool,
                                  const int*, std::vector<double>*);
template fm_status solve_core<float>(fm_plan*, int, const fm_solve_opts&, std::vector<fm_solve_info>&);
template fm_status solve_core<double>(fm_plan*, int, const fm_solve_opts&, std::vector<fm_solve_info>&);
template cudaError_t block_kernels<float, double>(fm_plan*, int, int, int, int, const void*, const void*, void*,
                                                  const int*, int, const int*);
template cudaError_t block_kernels<double, double>(fm_plan*, int, int, int, int, const void*, const void*, void*,
                                                   const int*, int, const int*);
template cudaError_t block_kernels<float, float>(fm_plan*, int, int, int, int, const void*, const void*, void*,
                                                 const int*, int, const int*);
