// libfmcuda: phantom permittivities painted on the device (phantoms.jl:58-362).
//
// The reference builds its phantoms on the host: a background array, then spheres (_fill_sphere!, :212-247),
// plates (phantom_plate, :156-199) or cylinders (_fill_cylinder!, :315-362) written into it in order.  Here the
// shapes become a small table and one kernel paints every voxel: the background, then each shape that covers the
// voxel, in table order, so a later shape overwrites an earlier one as in the reference's sequential fills.
//
// Exactness: a voxel is inside a shape by the reference's own tests, in FP64 and without fused multiply-adds, so
// the painted array equals the host one bit for bit:
//   sphere   bounding box [max(1, round(c - r)), min(N, round(c + r))] per axis (round: nearest, ties to even),
//            then dx*dx + dy*dy + dz*dz <= r^2 summed in that order (dx = i - c, 1-based i);
//   plate    [max(1, round(c - t/2)), min(N, round(c + t/2))] along its normal, the whole extent across;
//   cylinder [max(1, round(c - h/2)), min(N, round(c + h/2))] along its axis, and du*du + dv*dv <= r^2 over the
//            two other axes in increasing axis order.
#include <cfenv>
#include <cmath>

#include "fm_plan.cuh"

namespace {

struct ShapeDev {
  int lo[3], hi[3];   // inclusive 1-based box
  int radial;         // 0: box only (plate), 3: sphere, 1..3 + 4: cylinder along axis (radial - 4)
  double c[3];        // centre (1-based voxel coordinates)
  double r2;          // radius squared
  double2 value;
};

constexpr int kShapesPerBlock = 256;  // shapes staged in shared memory per pass

__device__ __forceinline__ double sq(double a) { return __dmul_rn(a, a); }

__global__ void __launch_bounds__(256) k_phantom_fill(int gx, int gy, int gz, double2 bg, int nshapes,
                                                      const ShapeDev* __restrict__ shapes, double2* __restrict__ eps) {
  __shared__ ShapeDev sh[kShapesPerBlock];
  const long long n = (long long)gx * gy * gz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  // every thread of the grid visits the same number of loop trips so that the block-wide staging stays uniform
  const long long trips = (n + stride - 1) / stride;
  for (long long t = 0; t < trips; ++t) {
    const long long idx = t * stride + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = idx < n;
    int i = 0, j = 0, k = 0;
    if (in) {
      i = (int)(idx % gx) + 1;
      const long long q = idx / gx;
      j = (int)(q % gy) + 1;
      k = (int)(q / gy) + 1;
    }
    double2 v = bg;
    for (int s0 = 0; s0 < nshapes; s0 += kShapesPerBlock) {
      const int cnt = min(kShapesPerBlock, nshapes - s0);
      __syncthreads();
      for (int q = threadIdx.x; q < cnt; q += blockDim.x) sh[q] = shapes[s0 + q];
      __syncthreads();
      if (!in) continue;
      for (int q = 0; q < cnt; ++q) {
        const ShapeDev& s = sh[q];
        if (i < s.lo[0] || i > s.hi[0] || j < s.lo[1] || j > s.hi[1] || k < s.lo[2] || k > s.hi[2]) continue;
        bool hit = true;
        if (s.radial == 3) {
          const double d = __dadd_rn(__dadd_rn(sq((double)i - s.c[0]), sq((double)j - s.c[1])), sq((double)k - s.c[2]));
          hit = d <= s.r2;
        } else if (s.radial >= 4) {
          const int ax = s.radial - 4;
          const double du = ax == 0 ? (double)j - s.c[1] : (double)i - s.c[0];
          const double dv = ax == 2 ? (double)j - s.c[1] : (double)k - s.c[2];
          hit = __dadd_rn(sq(du), sq(dv)) <= s.r2;
        }
        if (hit) v = s.value;
      }
    }
    if (in) eps[idx] = v;
  }
}

// round(Int, x) of the reference: nearest, ties to even
int round_even(double x) {
  const int old = std::fegetround();
  std::fesetround(FE_TONEAREST);
  const double r = std::nearbyint(x);
  std::fesetround(old);
  return (int)r;
}

}  // namespace

fm_status fm_phantom_fill(fm_plan* P, double eps_bg, int nshapes, const fm_shape* shapes, double* eps_out) {
  if (!P) return fail(FM_ERR_INVALID, "null plan");
  if (!(eps_bg > 0)) return fail(FM_ERR_INVALID, "permittivity_bg must be positive");
  if (nshapes < 0 || (nshapes > 0 && !shapes)) return fail(FM_ERR_INVALID, "bad shape list");
  FM_CK(cudaSetDevice(P->desc.device));
  const int g[3] = {P->pi.gx, P->pi.gy, P->pi.gz};
  std::vector<ShapeDev> tab;
  tab.reserve(nshapes);
  for (int q = 0; q < nshapes; ++q) {
    const fm_shape& s = shapes[q];
    if (!std::isfinite(s.value[0]) || !std::isfinite(s.value[1])) return fail(FM_ERR_NONFINITE, "shape permittivity");
    ShapeDev d{};
    for (int a = 0; a < 3; ++a) {
      d.c[a] = s.center[a];
      d.lo[a] = 1;
      d.hi[a] = g[a];
    }
    d.value = make_double2(s.value[0], s.value[1]);
    if (s.kind == FM_SHAPE_SPHERE) {
      if (!(s.radius > 0)) return fail(FM_ERR_INVALID, "pixel_radius must be positive");
      for (int a = 0; a < 3; ++a) {
        d.lo[a] = std::max(1, round_even(s.center[a] - s.radius));
        d.hi[a] = std::min(g[a], round_even(s.center[a] + s.radius));
      }
      d.radial = 3;
      d.r2 = s.radius * s.radius;
    } else if (s.kind == FM_SHAPE_PLATE || s.kind == FM_SHAPE_CYLINDER) {
      if (s.axis < 1 || s.axis > 3) return fail(FM_ERR_INVALID, "axis must be 1, 2, or 3");
      if (!(s.extent > 0)) return fail(FM_ERR_INVALID, "thickness / height must be positive");
      const int a = s.axis - 1;
      d.lo[a] = std::max(1, round_even(s.center[a] - s.extent / 2));
      d.hi[a] = std::min(g[a], round_even(s.center[a] + s.extent / 2));
      if (s.kind == FM_SHAPE_CYLINDER) {
        if (!(s.radius > 0)) return fail(FM_ERR_INVALID, "radius_pixel must be positive");
        d.radial = 4 + a;
        d.r2 = s.radius * s.radius;
      }
    } else {
      return fail(FM_ERR_INVALID, "unknown shape kind");
    }
    tab.push_back(d);
  }
  const long long n = (long long)g[0] * g[1] * g[2];
  FM_CK(P->eps_dev.ensure((size_t)n * sizeof(double2)));
  DevBuf& shp = P->shapes;
  FM_CK(shp.ensure(std::max<size_t>(16, tab.size() * sizeof(ShapeDev))));
  if (!tab.empty())
    FM_CK(cudaMemcpyAsync(shp.p, tab.data(), tab.size() * sizeof(ShapeDev), cudaMemcpyHostToDevice, P->st));
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)P->sms * 8);
  FM_TRACK(P, KC_SETUP, (double)n * sizeof(double2),
           (k_phantom_fill<<<blocks, 256, 0, P->st>>>(g[0], g[1], g[2], make_double2(eps_bg, 0.0), (int)tab.size(),
                                                       (const ShapeDev*)shp.p, (double2*)P->eps_dev.p)));
  FM_CK(cudaGetLastError());
  if (eps_out)
    FM_CK(cudaMemcpyAsync(eps_out, P->eps_dev.p, (size_t)n * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  FM_CK(cudaStreamSynchronize(P->st));
  P->eps_phantom = true;
  return FM_OK;
}
