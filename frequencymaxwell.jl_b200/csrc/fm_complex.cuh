// Complex arithmetic on float2 / double2 for the fmcuda kernels.
#pragma once
#include <cuda_runtime.h>
#include <type_traits>

namespace fm {

template <typename R> struct CT;
template <> struct CT<float>  { using T = float2; };
template <> struct CT<double> { using T = double2; };
template <typename R> using cplx = typename CT<R>::T;

template <typename T> struct RealOf;
template <> struct RealOf<float2>  { using R = float; };
template <> struct RealOf<double2> { using R = double; };

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <typename T> __host__ __device__ __forceinline__ T cadd(T a, T b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T> __host__ __device__ __forceinline__ T csub(T a, T b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T> __host__ __device__ __forceinline__ T cmul(T a, T b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T> __host__ __device__ __forceinline__ T cmulc(T a, T b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T> __host__ __device__ __forceinline__ T cconj(T a) { return mk(a.x, -a.y); }
template <typename T, typename R> __host__ __device__ __forceinline__ T cscale(T a, R s) { return mk(a.x * s, a.y * s); }
// multiply by i*sgn  (sgn = +1 -> i, -1 -> -i)
template <int SGN, typename T> __host__ __device__ __forceinline__ T cmul_i(T a) {
  return SGN > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
template <typename T> __host__ __device__ __forceinline__ T cinv(T a) {
  auto d = a.x * a.x + a.y * a.y;
  return mk(a.x / d, -a.y / d);
}
template <typename T> __host__ __device__ __forceinline__ T czero() { return mk(decltype(T{}.x)(0), decltype(T{}.x)(0)); }

__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <typename T> __device__ __forceinline__ T from_d(double2 a);
template <> __device__ __forceinline__ float2 from_d<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }

}  // namespace fm
