// libfmcuda: the Green application / CBS operator and the curl on device buffers -- the fused axis passes
// (fm_passes.cuh, fm_passes_tma.cuh) or the general passes (fm_generic.cuh) -- for every plan kind.
#include "fm_plan.cuh"

// ---------------------------------------------------------------------------
// Green application / CBS operator on device buffers (plan precision)
//   in  : nb fields
//   out : nb fields (may not alias in, t1, t2)
//   pro : PRO_COPY (psi = in) or PRO_V / PRO_V_SCALE (psi = V.*in [* scale])
//   epi : EPI_* epilogue applied to g = G_avg(psi)
// ---------------------------------------------------------------------------

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
fm_status green_op(fm_plan* P, int nb, const void* in, int pro, const double* rs, int epi, const void* xv,
                   const void* bv, const EpiParams& ep_in, void* out, const int* act, int nact, const RhsCtx* rc,
                   int chain) {
  using T = cplx<R>;
  if (chain) {
    if (!green_chain_ok(P, rc) || ((chain & GREEN_CHAIN_HAVE_XF) && pro != PRO_V) ||
        ((chain & GREEN_CHAIN_NEXT_XF) && (epi != EPI_PREC_OP || rs || xv != in)))
      return fail(FM_ERR_INVALID, "operator chaining needs the fused passes, PRO_V and EPI_PREC_OP on the input");
  }
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
    if (!(chain & GREEN_CHAIN_HAVE_XF)) {
      FM_TRACK(P, KC_XF, 2 * fbA + (pro != PRO_COPY ? vb : 0.0),
               e = pass_xf<R>(P, d, pro, in, V, rs, P->twx.p, nullptr, P->t1.p, act, vt));
      FM_CK(e);
    }
    FM_TRACK(P, KC_YF, 2 * fbA, e = pass_y<R>(P, d, -1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_ZG, 2 * fbA,
             e = pass_zg<R>(P, d, mode, P->t2.p, gp, P->zonly ? P->twz2.p : P->twz.p, P->zonly ? P->rz.p : nullptr,
                              P->t1.p, act));
    FM_CK(e);
    FM_TRACK(P, KC_YI, 2 * fbA, e = pass_y<R>(P, d, +1, P->t1.p, P->twy.p, nullptr, P->t2.p, act));
    FM_CK(e);
    if (chain & GREEN_CHAIN_NEXT_XF)
      FM_TRACK(P, KC_XI, xib + fbA, e = pass_xi_xf<R>(P, d, P->t2.p, V, xv, ep, P->twx.p, out, P->t1.p, act));
    else
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

// H = -i lambda/(2 pi 377) curl(E) for nb fields (in -> out, both contiguous batches; act masks RHS)
template <typename R>
fm_status curl_batch(fm_plan* P, int nb, const void* in, void* out, const int* act) {
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

template fm_status green_op<float>(fm_plan*, int, const void*, int, const double*, int, const void*, const void*,
                                   const EpiParams&, void*, const int*, int, const RhsCtx*, int);
template fm_status green_op<double>(fm_plan*, int, const void*, int, const double*, int, const void*, const void*,
                                    const EpiParams&, void*, const int*, int, const RhsCtx*, int);
template fm_status curl_batch<float>(fm_plan*, int, const void*, void*, const int*);
template fm_status curl_batch<double>(fm_plan*, int, const void*, void*, const int*);
