// libfmcuda: the C ABI (include/fmcuda.h) -- plan lifetime, potential set-up, the reference seams on host
// buffers, plane-wave solves with their output copies, instrumentation and tuning.
#include "fm_plan.cuh"

thread_local std::string g_err;

namespace fm {
// lets other translation units of the library report through fm_last_error()
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace fm

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
                    &P->gkn[0][1], &P->gkn[1][0], &P->gkn[1][1], &P->gkn[2][0], &P->gkn[2][1], &P->shapes};
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

void set_scalars(fm_plan* P, double k_bg, double eps_imag, double wavelength) {
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
  if (eps) {  // else the permittivity fm_phantom_fill painted on the device
    FM_CK(P->eps_dev.ensure((size_t)g * sizeof(double2)));
    FM_CK(cudaMemcpyAsync(P->eps_dev.p, eps, (size_t)g * sizeof(double2), cudaMemcpyHostToDevice, P->st));
    P->eps_phantom = false;
  }
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
  if (!eps && !P->eps_phantom) return fail(FM_ERR_INVALID, "null permittivity and no device phantom (fm_phantom_fill)");
  if (!(eps_bg > 0)) return fail(FM_ERR_INVALID, "permittivity_bg must be positive");
  if (!(wl > 0)) return fail(FM_ERR_INVALID, "wavelength must be positive");
  return P->prec == FM_PREC_F64 ? build_potential_t<double>(P, eps, eps_bg, wl, fx, fy, fz, itmax, info)
                                : build_potential_t<float>(P, eps, eps_bg, wl, fx, fy, fz, itmax, info);
}

// Plane-wave tables (FP64) of one source, following generate_incident_field
// (sources.jl): per-axis phase tables exp(i k_b k_d r_d) over the padded axis
// (source amplitude and phase folded into the z table) and the E and H
// polarisations.  tx/ty/tz have nx/ny/nz entries, pe/ph three each.
fm_status wave_tables(const fm_plan* P, const fm_plane_wave& w, double eps_bg, double2* tx, double2* ty,
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
      if (value < 0 || value > 2) return fail(FM_ERR_INVALID, "block-dot tuning value must be 0, 1 or 2");
      P->bd_bulk = value == 1;
      P->bd_wide = value == 2;
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
    case FM_TUNE_BLOCK_DOT: *value = P->bd_bulk ? 1 : P->bd_wide ? 2 : 0; return FM_OK;
    default: return fail(FM_ERR_INVALID, "unknown tuning knob");
  }
}

