/* fmcuda.h -- C ABI of libfmcuda, the B200 (sm_100a) convergent Born series solver.
 *
 * The library replaces the device path of FrequencyMaxwell.jl's
 * solve(solver::ConvergentBornSolver, sources, medium): the KernelAbstractions
 * kernels, the FFTW/CUFFT transforms and the LinearSolve/Krylov loop.  Host code
 * (Julia via ccall, Python via ctypes) keeps the reference API and calls these
 * entry points.  Each function names the reference code it stands in for
 * (paths inside the FrequencyMaxwell.jl project).
 *
 * Conventions
 *   - Complex arrays cross the ABI as interleaved FP64 (re, im) pairs.
 *   - Fields are column-major (Nx', Ny', Nz', 3) per right-hand side (RHS), x
 *     fastest, components planar, RHS outermost: element (x,y,z,c,b) at
 *     x + Nx'*(y + Ny'*(z + Nz'*(c + 3*b))).  Nx', Ny', Nz' are the padded sizes.
 *   - A plan owns all device memory and one CUDA stream.  Plans are not
 *     thread-safe; different plans may be used from different host threads.
 *   - Every entry point returns an fm_status; fm_last_error() gives a message
 *     for the calling thread.  Non-convergence returns FM_NOT_CONVERGED with the
 *     result still written (the reference only warns:
 *     src/solvers/convergent_born.jl:753-755).
 */
#ifndef FMCUDA_H
#define FMCUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define FMCUDA_ABI_VERSION 2

typedef enum {
  FM_OK = 0,
  FM_ERR_INVALID = 1,      /* bad argument (reference: ArgumentError) */
  FM_ERR_OOM = 2,          /* device allocation failed */
  FM_NOT_CONVERGED = 3,    /* iteration limit reached; outputs written */
  FM_ERR_NONFINITE = 4,    /* NaN/Inf found in an input or a result */
  FM_ERR_TIMEOUT = 5,      /* host-side deadline passed */
  FM_ERR_CUDA = 6,         /* CUDA runtime error */
  FM_ERR_UNSUPPORTED = 7   /* size or option this build does not support */
} fm_status;

/* FM_PREC_F32_MATH64: fields stored as complex FP32 in HBM (FP32 traffic), FFT / Green / potential
 * arithmetic carried out in FP64 registers. */
enum { FM_PREC_F64 = 0, FM_PREC_F32 = 1, FM_PREC_F32_MATH64 = 2 };
enum { FM_METHOD_GMRES = 0, FM_METHOD_BICGSTAB = 1, FM_METHOD_RICHARDSON = 2 };
/* FM_ORTHO_BLOCK: s-step GMRES.  The first `block` iterations are classical Gram-Schmidt; after them each
 * step builds `block` Krylov vectors with Newton shifts (Ritz values of the first steps) and orthogonalises
 * them together against the basis, so the basis is read twice per `block` iterations instead of twice per
 * iteration.  The Hessenberg matrix is recovered exactly from the block relations, so in exact arithmetic
 * the iterate, residual estimates and stopping iteration are those of full GMRES.  Full GMRES only
 * (restart = 0). */
enum { FM_ORTHO_MGS = 0, FM_ORTHO_CGS = 1, FM_ORTHO_CGS2 = 2, FM_ORTHO_BLOCK = 3 };
/* FM_ORTHO_BLOCK: type of the raw block vectors before they are orthogonalised.  FM_BLOCK_FP64 keeps them in
 * complex FP64 on plans that compute in FP64 (FM_PREC_F64, FM_PREC_F32_MATH64), which keeps the accuracy of
 * classical Gram-Schmidt; FM_BLOCK_STORAGE keeps them in the plan's storage type (less traffic, larger
 * rounding error on FP32-storage plans).  FM_BLOCK_FP64_ORTHO is FM_BLOCK_FP64 that also keeps the projected
 * block in FP64 and stores it orthonormalised (V = Y' Rb^{-1}) instead of raw: the rounding of the stored basis
 * is then not amplified by the condition number of the block, at the cost of one more pass over the S new
 * vectors per block. */
enum { FM_BLOCK_FP64 = 0, FM_BLOCK_STORAGE = 1, FM_BLOCK_FP64_ORTHO = 2 };

typedef struct fm_plan fm_plan;

/* Grid description.  Mirrors what ConvergentBornSolver derives from its
 * boundary conditions: padding_pixels and subpixel_shift per axis
 * (src/solvers/boundary_conditions.jl:450-527) and compute_ROI
 * (src/solvers/convergent_born.jl:250-260). */
typedef struct {
  int grid[3];          /* unpadded (Nx, Ny, Nz) */
  int pad[3];           /* padding pixels per side and axis */
  double resolution[3]; /* voxel size in metres */
  int absorbing[3];     /* 1: absorbing axis -> shift 0.25 and (G(+s)+G(-s))/2 averaging */
  int precision;        /* FM_PREC_F64, FM_PREC_F32 or FM_PREC_F32_MATH64 */
  int max_rhs;          /* largest batch the plan will be asked to hold at once (>= 1) */
  int device;           /* CUDA device ordinal */
} fm_plan_desc;

typedef struct {
  int method;           /* FM_METHOD_* (reference default: GMRES, convergent_born.jl:197) */
  int ortho;            /* FM_ORTHO_* for GMRES (Krylov.jl uses MGS) */
  int restart;          /* 0: full GMRES as KrylovJL_GMRES runs it; m > 0: GMRES(m) */
  int maxiters;         /* max(2*Bornmax, 100) in the reference (convergent_born.jl:746) */
  double reltol;        /* solver.tolerance (convergent_born.jl:744) */
  double abstol;        /* solver.tolerance * 1e-2 (convergent_born.jl:745) */
  double timeout_s;     /* host-side deadline for the whole call, 0 = none */
  int block;            /* FM_ORTHO_BLOCK: vectors per block, 2..8 (0: 4); ignored otherwise */
  int block_store;      /* FM_ORTHO_BLOCK: FM_BLOCK_FP64, FM_BLOCK_STORAGE or FM_BLOCK_FP64_ORTHO; ignored otherwise */
} fm_solve_opts;

typedef struct {
  int iterations;       /* Krylov iterations (sol.iters, convergent_born.jl:761-763) */
  int solved;           /* 1 when the stopping test was met */
  double residual;      /* last preconditioned residual estimate (sol.resid, :764-766) */
  double residual0;     /* initial preconditioned residual norm */
} fm_solve_info;

typedef struct {
  double eps_imag;      /* max(2^-20, 1.01 max|V|)   (convergent_born.jl:641) */
  double k_bg;          /* 2 pi sqrt(eps_bg) / lambda (convergent_born.jl:630) */
  int bornmax;          /* Bornmax (convergent_born.jl:653-660) */
} fm_potential_info;

/* One plane-wave source, as PlaneWaveSource holds it (src/sources/plane_wave.jl:63-116). */
typedef struct {
  double wavelength;
  double polarization[6];  /* 3 complex values, interleaved (re, im) */
  double k_vector[3];      /* unit propagation direction */
  double amplitude;
  double phase;
} fm_plane_wave;

int fm_abi_version(void);
const char* fm_last_error(void);
int fm_device_count(void);

/* Plan lifetime.  Replaces the device-side state that ConvergentBornSolver and
 * DyadicGreen allocate per solve (convergent_born.jl:619-675,
 * src/core/dyadic_green.jl:67-99). */
fm_status fm_plan_create(const fm_plan_desc* desc, fm_plan** out);
void fm_plan_destroy(fm_plan* plan);
/* Device bytes a plan needs to hold `nrhs` right-hand sides with a Krylov basis of `basis` vectors. */
long long fm_plan_bytes(const fm_plan_desc* desc, int nrhs, int basis);

/* ---- reference seams (host buffers) ------------------------------------ */

/* to_device(V) of _initialize_solver! (convergent_born.jl:649-650): the padded,
 * attenuated potential including the -i*eps_imag shift, plus the scalars that
 * the reference derives next to it. */
fm_status fm_set_potential(fm_plan* plan, const double* V, double k_bg, double eps_imag, double wavelength);

/* conv!(::DyadicGreen, x) (src/core/dyadic_green.jl:127-152), nrhs fields in, nrhs fields out. */
fm_status fm_green_apply(fm_plan* plan, int nrhs, const double* x, double* y);

/* mul!(y, ::CBSLinearOperator, x, alpha, beta): y = beta*y + alpha*(x - G_avg(V.*x))
 * (convergent_born.jl:482-512). */
fm_status fm_apply_operator(fm_plan* plan, int nrhs, const double* x, double* y, double alpha_re, double alpha_im,
                            double beta_re, double beta_im);

/* ldiv!(y, ::CBSPreconditioner, x): y = (i/eps_imag) .* V .* x (convergent_born.jl:398-410). */
fm_status fm_apply_preconditioner(fm_plan* plan, int nrhs, const double* x, double* y);

/* _compute_magnetic_field (convergent_born.jl:784-800 with src/core/curl.jl:55-116):
 * H = -i*lambda/(2*pi*377) * curl(E). */
fm_status fm_curl_field(fm_plan* plan, int nrhs, const double* E, double* H);

/* _solve_cbs_scattering (convergent_born.jl:703-774): from source terms S (the
 * reference's V.*E_inc + i*eps_imag.*E_inc, :585-586) to the scattered E and H on
 * the padded grid.  info is an array of nrhs entries. */
fm_status fm_solve_source(fm_plan* plan, int nrhs, const double* S, const fm_solve_opts* opts, double* E_scat,
                          double* H_scat, fm_solve_info* info);

/* ---- device-side set-up and assembly ----------------------------------- */

/* The numerics of _initialize_solver! (convergent_born.jl:625-660) run on the
 * device from the unpadded permittivity (Nx, Ny, Nz) complex array.  fx, fy, fz
 * are the per-axis attenuation filters over the padded axes (all ones on
 * periodic axes), as _apply_attenuation_to_potential! builds them
 * (convergent_born.jl:893-944).  eps = NULL takes the permittivity that fm_phantom_fill painted on the
 * device. */
fm_status fm_build_potential(fm_plan* plan, const double* eps, double eps_bg, double wavelength, const double* fx,
                             const double* fy, const double* fz, int iterations_max, fm_potential_info* info);

/* ---- phantoms painted on the device (phantoms.jl:58-362) ----
 * The reference's phantom generators fill a host array: the background, then spheres (_fill_sphere!,
 * phantoms.jl:212-247: bounding box [max(1, round(c - r)), min(N, round(c + r))] per axis, then
 * (i-c1)^2 + (j-c2)^2 + (k-c3)^2 <= r^2 with 1-based indices), plates (phantom_plate, :156-199: the slab
 * [max(1, round(c - t/2)), min(N, round(c + t/2))] along its normal) and cylinders (phantom_cylinder /
 * _fill_cylinder!, :272-362: that range along the axis, and the squared distance over the two other axes
 * <= r^2).  fm_phantom_fill paints the same shapes, in order (later shapes overwrite earlier ones), into the
 * plan's device permittivity (grid_size, complex FP64) with the same FP64 tests, bit for bit; the next
 * fm_build_potential with eps = NULL builds the potential from it, so no permittivity crosses from the host.
 * eps_out (optional, host, (Nx, Ny, Nz) complex FP64) receives a copy.  `round` is to nearest, ties to even. */
enum { FM_SHAPE_SPHERE = 0, FM_SHAPE_PLATE = 1, FM_SHAPE_CYLINDER = 2 };
typedef struct {
  int kind;             /* FM_SHAPE_* */
  int axis;             /* plate normal / cylinder axis, 1..3 (spheres: unused) */
  double center[3];     /* 1-based voxel coordinates; (N+1)/2 is the grid centre as in the reference */
  double radius;        /* sphere / cylinder radius in pixels */
  double extent;        /* plate thickness / cylinder height in pixels */
  double value[2];      /* permittivity (re, im) */
} fm_shape;
fm_status fm_phantom_fill(fm_plan* plan, double permittivity_bg, int nshapes, const fm_shape* shapes,
                          double* eps_out);

/* The whole of solve(solver, sources, medium) after set-up (convergent_born.jl:576-599):
 * incident plane waves (generate_incident_field, plane_wave.jl:198-268, coherent sum
 * field_generation.jl:42-78), source term, CBS solve, magnetic field, incident
 * addition and crop_to_ROI.  RHS b owns sources [first[b], first[b+1]).  E_out and
 * H_out receive the cropped total fields (Nx, Ny, Nz, 3) per RHS; when they are
 * NULL the fields stay on the device (see fm_copy_fields). */
fm_status fm_solve_plane_waves(fm_plan* plan, int nrhs, const int* first, const fm_plane_wave* sources,
                               double permittivity_bg, const fm_solve_opts* opts, double* E_out, double* H_out,
                               fm_solve_info* info);

/* Copy the cropped total fields of the last fm_solve_plane_waves call to the host. */
fm_status fm_copy_fields(fm_plan* plan, int nrhs, double* E_out, double* H_out);

/* Wait for the plan's stream. */
fm_status fm_synchronize(fm_plan* plan);

/* ---- continuous batching: the slot engine ----------------------------------
 * No counterpart in the reference (it solves one request per call).  An engine owns `slots` right-hand
 * sides on one plan; each slot holds one plane-wave right-hand side on its own permittivity, with its own
 * potential, eps_imag, Krylov basis of up to `basis` vectors and GMRES state (the reference's
 * KrylovJL_GMRES semantics per right-hand side: warm start b, maxiters = max(2*Bornmax, 100), reltol =
 * tolerance, abstol = tolerance*1e-2; when maxiters exceeds `basis` the slot restarts GMRES every `basis`
 * iterations, i.e. it runs GMRES(basis), and full GMRES as the reference when maxiters fits the basis).  Requests share the engine's
 * wavelength, background permittivity and attenuation filters (fx, fy, fz over the padded axes, NULL =
 * ones) and take over the plan.  ortho: FM_ORTHO_CGS, FM_ORTHO_CGS2, or FM_ORTHO_BLOCK, with which the slots
 * run s-step block GMRES (s = 8, FP64 block vectors stored orthonormalised, as fm_solve with FM_ORTHO_BLOCK and
 * FM_BLOCK_FP64_ORTHO; needs basis >= 16 and 3 x padded voxels a multiple of 4, else CGS): full GMRES when
 * maxiters + 8 <= basis, otherwise restarted every floor(basis / 8) * 8 iterations.  fm_engine_step admits queued
 * right-hand sides into free slots, runs one Krylov iteration (a block slot: one block of 8 after the first 8
 * iterations of a cycle) on every running slot in shared launches (slots at different iterations), and
 * finishes the slots that stopped: their cropped total E and H are copied to the caller's host buffers
 * given at submission (nrhs x (Nx,Ny,Nz,3) complex FP64 each), which must stay valid until then.
 * fm_engine_submit may be called from another thread than fm_engine_step. */
typedef struct fm_engine fm_engine;
/* Device bytes one slot needs (basis vectors + work + outputs). */
long long fm_engine_slot_bytes(const fm_plan_desc* desc, int basis);
/* The same for an engine created with `ortho` (FM_ORTHO_BLOCK adds the block vectors of block GMRES). */
long long fm_engine_slot_bytes_ortho(const fm_plan_desc* desc, int basis, int ortho);
fm_status fm_engine_create(fm_plan* plan, int slots, int basis, double wavelength, double permittivity_bg,
                           const double* fx, const double* fy, const double* fz, int ortho, fm_engine** out);
void fm_engine_destroy(fm_engine* engine);
fm_status fm_engine_submit(fm_engine* engine, long long request_id, const double* eps, int nrhs,
                           const fm_plane_wave* sources, double tolerance, int iterations_max, double* E_out,
                           double* H_out);
/* Completed right-hand sides of this step: request id, index within the request and solve info. */
fm_status fm_engine_step(fm_engine* engine, int* n_done, long long* done_request, int* done_rhs,
                         fm_solve_info* done_info, int max_done);
fm_status fm_engine_status(fm_engine* engine, int* running, int* queued);

/* ---- Green application without device allocation ----------------------
 * No counterpart in the reference.  For callers that cannot let a library call cudaMalloc (their own
 * pooled allocator, a fixed device-memory budget, a loop that must not touch the allocator): the
 * Green application conv!(G, x) of fm_green_apply on device buffers the caller owns, with no plan.
 * x_dev and y_dev hold nrhs fields in the storage type of desc->precision (complex128 for
 * FM_PREC_F64, complex64 otherwise), laid out as above; they must not overlap (y doubles as a pass
 * temporary).  desc gives grid, padding, resolution, boundaries, precision and device; max_rhs is
 * ignored.  The only scratch is one static 64 MiB device array per GPU that loads the library
 * (tables, an error flag and one field-sized temporary), so sizes whose temporary does not fit are
 * rejected with FM_ERR_INVALID.  The first call on a device looks up that array's address.  Calls share
 * the array: calls that overlap on the GPU race.  Work is
 * issued on `stream` (NULL: default stream) and the call returns after it has finished. */
fm_status fm_green_apply_noalloc(const fm_plan_desc* desc, double k_bg, double eps_imag, int nrhs, const void* x_dev,
                                 void* y_dev, void* stream);

/* ---- instrumentation (no reference counterpart: measurement support) ---- */

typedef struct {
  char name[16];        /* kernel class: xf, yf, zg, yi, xi, multidot, update, mgs, axpby, curl, setup */
  long long launches;   /* launches since the last fm_set_profiling */
  double ms;            /* summed device time from CUDA events on the plan stream (profiling on) */
  double bytes;         /* summed algorithmic HBM bytes of those launches */
} fm_kernel_stat;

/* Reset the counters; on != 0 also brackets every launch with CUDA events on the plan's stream. */
fm_status fm_set_profiling(fm_plan* plan, int on);
/* Fill up to max entries (one per kernel class); returns the number written. */
int fm_kernel_stats(fm_plan* plan, fm_kernel_stat* out, int max);
/* Kernel launches issued by the plan since the last fm_set_profiling. */
long long fm_launch_count(fm_plan* plan);
/* The plan's cudaStream_t, for callers that time work on it with their own events. */
void* fm_stream(fm_plan* plan);

/* Launch-shape and batch-schedule knobs of a plan, set by the autotuner (fmcuda/autotune.py).  They change
 * how work is launched, never what is computed.  No counterpart in the reference.
 *   FM_TUNE_Y_TMA, FM_TUNE_Z_TMA    1: TMA-staged y / z passes where the axis length has one, 0: register-only
 *   FM_TUNE_TMA_CTAS_PER_SM         persistent CTAs per SM of the TMA passes, 0 = occupancy limit
 *   FM_TUNE_ROW_THREADS             threads per block of the x and y row passes: 128 or 256
 *   FM_TUNE_WAVE_RHS                right-hand sides per wave at most, 0 = as many as device memory holds
 *   FM_TUNE_BLOCK_DOT               block dot of block GMRES: 0 = the register-staged kernel, 1 = bulk-copy
 *                                   pipeline (one CTA per SM), 2 = the register-staged kernel with four groups of
 *                                   basis vectors per warp (blocks of 5..8 vectors) */
enum { FM_TUNE_Y_TMA = 0, FM_TUNE_Z_TMA = 1, FM_TUNE_TMA_CTAS_PER_SM = 2, FM_TUNE_ROW_THREADS = 3,
       FM_TUNE_WAVE_RHS = 4, FM_TUNE_BLOCK_DOT = 5 };
fm_status fm_plan_set_tuning(fm_plan* plan, int knob, int value);
fm_status fm_plan_get_tuning(fm_plan* plan, int knob, int* value);

#ifdef __cplusplus
}
#endif
#endif /* FMCUDA_H */
