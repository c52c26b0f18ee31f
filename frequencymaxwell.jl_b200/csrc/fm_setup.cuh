// Device-side problem set-up and output assembly (FP64 arithmetic).
//
//  * potential: V = k_bg^2 (eps/eps_bg - 1) on the unpadded grid, zero padding,
//    eps_imag = max(2^-20, 1.01 max|V|), V -= i eps_imag, separable attenuation
//    filters per axis (identity on periodic axes), then scaled to the plan's
//    units (divided by k_ref^2) and stored in the plan precision.
//  * source term: S = (V + i eps_imag) .* E_inc with the incident plane-wave sum
//    evaluated from separable per-axis phase tables (exp(i k_d r_d) in FP64).
//  * output: total fields E = E_s + E_inc, H = H_s + H_inc cropped to the ROI,
//    assembled in FP64.
#pragma once
#include "fm_complex.cuh"

namespace fm {

// max |k^2 (eps/eps_bg - 1)| over the unpadded grid (deterministic two-level)
static __global__ void __launch_bounds__(256) k_potential_max(long long n, const double2* __restrict__ eps, double eps_bg,
                                                        double k2, double* __restrict__ part, double* __restrict__ out,
                                                        unsigned* __restrict__ counter) {
  __shared__ double red[8];
  __shared__ bool last;
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 e = eps[i];
    double vr = k2 * (e.x / eps_bg - 1.0), vi = k2 * (e.y / eps_bg);
    m = fmax(m, hypot(vr, vi));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = fmax(t, red[q]);
    part[blockIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned k = 0; k < gridDim.x; ++k) t = fmax(t, __ldcg(&part[k]));
    *out = t;
    *counter = 0;
  }
}

struct PadInfo {
  int gx, gy, gz;   // unpadded
  int px, py, pz;   // padding per side
  int nx, ny, nz;   // padded
};

// V (padded, plan precision, scaled by inv_kref2)
template <typename R>
__global__ void __launch_bounds__(256) k_potential_build(PadInfo pi, const double2* __restrict__ eps, double eps_bg,
                                                          double k2, double eps_imag, const double* __restrict__ fx,
                                                          const double* __restrict__ fy, const double* __restrict__ fz,
                                                          double inv_kref2, cplx<R>* __restrict__ V) {
  const long long n = (long long)pi.nx * pi.ny * pi.nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % pi.nx);
    const int y = (int)((i / pi.nx) % pi.ny);
    const int z = (int)(i / ((long long)pi.nx * pi.ny));
    const int ux = x - pi.px, uy = y - pi.py, uz = z - pi.pz;
    double vr = 0.0, vi = 0.0;
    if (ux >= 0 && ux < pi.gx && uy >= 0 && uy < pi.gy && uz >= 0 && uz < pi.gz) {
      double2 e = eps[ux + (long long)pi.gx * (uy + (long long)pi.gy * uz)];
      vr = k2 * (e.x / eps_bg - 1.0);
      vi = k2 * (e.y / eps_bg);
    }
    vi -= eps_imag;
    const double f = fx[x] * fy[y] * fz[z];
    V[i] = from_d<cplx<R>>(make_double2(vr * f * inv_kref2, vi * f * inv_kref2));
  }
}

// One plane wave of an RHS: per-axis phase tables and polarisations.
// ph[d] points to a table of exp(i k_d r_d) (the source phase and amplitude are
// folded into the z table) over the padded axis.
struct WaveTabs {
  const double2* tx;   // [nsrc_total][nx]
  const double2* ty;   // [nsrc_total][ny]
  const double2* tz;   // [nsrc_total][nz]
  const double2* pe;   // [nsrc_total][3]   E polarisation
  const double2* ph;   // [nsrc_total][3]   H polarisation
  const int* first;    // [B+1] source range of each RHS
};

__device__ __forceinline__ void incident_at(const WaveTabs& w, const PadInfo& pi, int b, int x, int y, int z,
                                            double2 (&E)[3], double2 (&H)[3], bool want_h) {
#pragma unroll
  for (int c = 0; c < 3; ++c) { E[c] = make_double2(0, 0); H[c] = make_double2(0, 0); }
  for (int s = w.first[b]; s < w.first[b + 1]; ++s) {
    double2 a = cmul(cmul(w.tx[(size_t)s * pi.nx + x], w.ty[(size_t)s * pi.ny + y]), w.tz[(size_t)s * pi.nz + z]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      E[c] = cadd(E[c], cmul(a, w.pe[s * 3 + c]));
      if (want_h) H[c] = cadd(H[c], cmul(a, w.ph[s * 3 + c]));
    }
  }
}

// S[b] = (V + i eps') .* E_inc  in scaled units (V already scaled, eps_s = eps_imag * inv_kref2)
// (vstride, eps_b): per-RHS potential V + b*vstride and eps_b[b] (0 / null: shared V, eps_s)
template <typename R>
__global__ void __launch_bounds__(256) k_source_term(PadInfo pi, int B, WaveTabs w, const cplx<R>* __restrict__ V,
                                                      double eps_s, cplx<R>* __restrict__ S, const int* __restrict__ active,
                                                      long long vstride = 0, const double* __restrict__ eps_b = nullptr) {
  const long long n = (long long)pi.nx * pi.ny * pi.nz;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % pi.nx);
    const int y = (int)((i / pi.nx) % pi.ny);
    const int z = (int)(i / ((long long)pi.nx * pi.ny));
    double2 E[3], H[3];
    incident_at(w, pi, b, x, y, z, E, H, false);
    double2 v = to_d(V[b * vstride + i]);
    v.y += eps_b ? eps_b[b] : eps_s;
#pragma unroll
    for (int c = 0; c < 3; ++c) S[((size_t)b * 3 + c) * n + i] = from_d<cplx<R>>(cmul(v, E[c]));
  }
}

// Total fields cropped to the ROI, FP64, layout (gx, gy, gz, 3) per RHS.
template <typename R>
__global__ void __launch_bounds__(256) k_assemble(PadInfo pi, int B, WaveTabs w, const cplx<R>* __restrict__ Es,
                                                   const cplx<R>* __restrict__ Hs, double2* __restrict__ Eo,
                                                   double2* __restrict__ Ho, const int* __restrict__ active = nullptr) {
  const long long n = (long long)pi.nx * pi.ny * pi.nz;
  const long long g = (long long)pi.gx * pi.gy * pi.gz;
  const int b = blockIdx.y;
  if (active && !active[b]) return;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < g; i += (long long)gridDim.x * blockDim.x) {
    const int ux = (int)(i % pi.gx);
    const int uy = (int)((i / pi.gx) % pi.gy);
    const int uz = (int)(i / ((long long)pi.gx * pi.gy));
    const int x = ux + pi.px, y = uy + pi.py, z = uz + pi.pz;
    const long long pidx = x + (long long)pi.nx * (y + (long long)pi.ny * z);
    double2 E[3], H[3];
    incident_at(w, pi, b, x, y, z, E, H, true);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Eo[((size_t)b * 3 + c) * g + i] = cadd(E[c], to_d(Es[((size_t)b * 3 + c) * n + pidx]));
      Ho[((size_t)b * 3 + c) * g + i] = cadd(H[c], to_d(Hs[((size_t)b * 3 + c) * n + pidx]));
    }
  }
}

// conversions between host FP64 interleaved arrays and plan-precision device arrays
template <typename R>
__global__ void k_from_f64(long long n, const double2* __restrict__ a, double s, cplx<R>* __restrict__ o) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 v = a[i];
    o[i] = from_d<cplx<R>>(make_double2(v.x * s, v.y * s));
  }
}
template <typename R>
__global__ void k_to_f64(long long n, const cplx<R>* __restrict__ a, double s, double2* __restrict__ o) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 v = to_d(a[i]);
    o[i] = make_double2(v.x * s, v.y * s);
  }
}

// finite check (counts non-finite entries)
template <typename R>
__global__ void k_count_nonfinite(long long n, const cplx<R>* __restrict__ a, unsigned long long* __restrict__ cnt) {
  unsigned long long c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 v = to_d(a[i]);
    if (!isfinite(v.x) || !isfinite(v.y)) ++c;
  }
  if (c) atomicAdd(cnt, c);
}

}  // namespace fm
