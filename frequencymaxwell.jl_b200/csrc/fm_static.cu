// fm_green_apply_noalloc: the dyadic Green application for callers that cannot allocate device memory.
//
// Who needs it: code that owns every device buffer itself and forbids a library from calling
// cudaMalloc -- a host runtime with its own pooled allocator (Julia's CUDA.jl arrays, a framework
// memory pool), a real-time loop that must not hit the allocator, or a process that runs under a
// fixed device-memory budget.  Such a caller passes device pointers for the input and the output
// fields and gets the Green application without any plan (plans allocate their tables and buffers).
//
// Scratch: one file-scope __device__ array of FM_NOALLOC_SCRATCH_BYTES (64 MiB) holds the twiddle and
// ramp tables, the error flag of the pipelined passes and one field-sized temporary.  Every GPU that
// loads the library keeps it until the process exits.  Its device address is looked up once per device
// (cudaGetSymbolAddress with that device current) on the first call that uses the device.  All calls
// share the array and it keeps the last call's
// contents, so calls that overlap on the GPU (different streams or threads) race; the error flag is
// cleared at the start of every call.  Sizes whose temporary and tables do not fit are rejected with
// FM_ERR_INVALID.  The output buffer doubles as the second pass temporary, so x and y must not overlap.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fmcuda.h"
#include "fm_launch.h"
#include "fm_tables.h"

using namespace fm;

namespace fm {
void set_last_error(const std::string& msg);  // defined next to fm_last_error (fm_capi.cu)
}

namespace {

constexpr size_t FM_NOALLOC_SCRATCH_BYTES = 64ull << 20;
constexpr int FM_NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[FM_NOALLOC_SCRATCH_BYTES];

void* g_scratch_addr[FM_NOALLOC_MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mutex;

// errors are reported through fm_last_error(), like every other entry point
fm_status noalloc_fail(fm_status s, const std::string& m) {
  fm::set_last_error(m);
  return s;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of the scratch array on the current device (set-up once per device).
cudaError_t scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lk(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

template <typename C>
cudaError_t put_table(unsigned char* dst, const std::vector<cd_t>& v, cudaStream_t st) {
  std::vector<C> h(v.size());
  for (size_t i = 0; i < v.size(); ++i) h[i] = mk((typename RealOf<C>::R)v[i].real(), (typename RealOf<C>::R)v[i].imag());
  return cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(C), cudaMemcpyHostToDevice, st);
}

bool pow2_in(int n, int lo, int hi) { return n >= lo && n <= hi && (n & (n - 1)) == 0; }

template <typename S, typename R>
fm_status run(const fm_plan_desc& dsc, double k_bg, double eps_imag, int nrhs, const void* x, void* y, cudaStream_t st,
              int dev) {
  using CR = cplx<R>;
  const int n3[3] = {dsc.grid[0] + 2 * dsc.pad[0], dsc.grid[1] + 2 * dsc.pad[1], dsc.grid[2] + 2 * dsc.pad[2]};
  const bool avg = dsc.absorbing[0] || dsc.absorbing[1] || dsc.absorbing[2];
  const bool zonly = dsc.absorbing[2] && !dsc.absorbing[0] && !dsc.absorbing[1];
  Dims d{n3[0], n3[1], n3[2], nrhs, (long long)n3[0] * n3[1] * n3[2]};
  // scratch layout: [error flag | tw x | tw y | tw z (length Lz of the z pass) | ramp z | field temporary]
  const int lz = zonly ? 2 * n3[2] : n3[2];
  const size_t o_err = 0;
  const size_t o_tx = 256;
  const size_t o_ty = o_tx + align256(2 * (size_t)n3[0] * sizeof(CR));
  const size_t o_tz = o_ty + align256(2 * (size_t)n3[1] * sizeof(CR));
  const size_t o_rz = o_tz + align256(2 * (size_t)lz * sizeof(CR));
  const size_t o_tmp = o_rz + align256((size_t)n3[2] * sizeof(CR));
  const size_t field = (size_t)nrhs * 3 * d.n * sizeof(cplx<S>);
  const size_t need = o_tmp + field;
  if (need > FM_NOALLOC_SCRATCH_BYTES)
    return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: this size needs " + std::to_string(need) +
                                            " bytes of scratch; the static scratch holds " +
                                            std::to_string(FM_NOALLOC_SCRATCH_BYTES) + " bytes");
  (void)avg;
  void* base = nullptr;
  cudaError_t e = scratch_address(dev, &base);
  if (e != cudaSuccess) return noalloc_fail(FM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  unsigned char* sc = (unsigned char*)base;
  int* err = (int*)(sc + o_err);
  // tables (FP64 on the host, cast to the arithmetic type)
  if ((e = cudaMemsetAsync(err, 0, sizeof(int), st)) != cudaSuccess ||
      (e = put_table<CR>(sc + o_tx, twiddles<R>(n3[0]), st)) != cudaSuccess ||
      (e = put_table<CR>(sc + o_ty, twiddles<R>(n3[1]), st)) != cudaSuccess ||
      (e = put_table<CR>(sc + o_tz, twiddles<R>(lz), st)) != cudaSuccess ||
      (e = put_table<CR>(sc + o_rz, ramp(n3[2], zonly ? 0.25 : 0.0, -1.0), st)) != cudaSuccess)
    return noalloc_fail(FM_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
  // k in units of k_bg (as the plans compute it), so |k|^2 - k_square stays O(1) in FP32 arithmetic:
  // k' = k / k_bg, k_square' = k_square / k_bg^2, and G' = k_bg^2 G.  The factor 1 / k_bg^2 that returns the
  // output to physical units is folded into the scale with the inverse-transform normalisation.
  const double kref2 = k_bg * k_bg, kr = k_bg;
  GreenParams gp{};
  for (int a = 0; a < 3; ++a) gp.dk[a] = 2.0 * M_PI / ((double)n3[a] * dsc.resolution[a]) / kr;
  gp.shift[2] = zonly ? 0.25 : 0.0;
  gp.ksq_re = 1.0;
  gp.ksq_im = eps_imag / kref2;
  gp.scale_re = 1.0 / ((double)d.n * (zonly ? 2.0 : 1.0) * kref2);
  const int mode = zonly ? ZMODE_AVG2 : ZMODE_ONE;
  void* tmp = sc + o_tmp;
  EpiParams ep{};
  // x -> y (x FFT) -> tmp (y FFT) -> y (z FFT, Green, inverse z FFT) -> tmp (inverse y FFT) -> y (inverse x FFT)
  auto ytma = [&](int dir, const void* in, void* out) -> cudaError_t {
    cudaError_t r = launch_y_tma<S, R>(d, dir, in, sc + o_ty, nullptr, out, nullptr, err, sms, st);
    if (r == cudaErrorNotSupported) r = launch_y<S, R>(d, dir, in, sc + o_ty, nullptr, out, nullptr, st);
    return r;
  };
  if ((e = launch_xf<S, R>(d, PRO_COPY, x, nullptr, nullptr, sc + o_tx, nullptr, y, nullptr, st)) != cudaSuccess ||
      (e = ytma(-1, y, tmp)) != cudaSuccess)
    return noalloc_fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  e = launch_zg_tma<S, R>(d, mode, tmp, gp, sc + o_tz, zonly ? (const void*)(sc + o_rz) : nullptr, y, nullptr, err, sms, st);
  if (e == cudaErrorNotSupported)
    e = launch_zg<S, R>(d, mode, tmp, gp, sc + o_tz, zonly ? (const void*)(sc + o_rz) : nullptr, y, nullptr, st);
  if (e != cudaSuccess || (e = ytma(+1, y, tmp)) != cudaSuccess ||
      (e = launch_xi<S, R>(d, EPI_STORE, tmp, nullptr, nullptr, nullptr, nullptr, ep, sc + o_tx, nullptr, y, nullptr,
                           st)) != cudaSuccess)
    return noalloc_fail(FM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  int code = 0;
  if ((e = cudaMemcpyAsync(&code, err, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return noalloc_fail(FM_ERR_CUDA, std::string("synchronize: ") + cudaGetErrorString(e));
  if (code) return noalloc_fail(FM_ERR_TIMEOUT, "a pipeline wait timed out on the device (code " + std::to_string(code) + ")");
  return FM_OK;
}

}  // namespace

fm_status fm_green_apply_noalloc(const fm_plan_desc* desc, double k_bg, double eps_imag, int nrhs, const void* x_dev,
                                 void* y_dev, void* stream) {
  if (!desc || !x_dev || !y_dev) return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: null argument");
  if (nrhs < 1) return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: nrhs must be >= 1");
  if (!(k_bg > 0) || !(eps_imag > 0)) return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: k_bg and eps_imag must be positive");
  int n3[3];
  for (int a = 0; a < 3; ++a) {
    if (desc->grid[a] <= 0 || desc->pad[a] < 0 || !(desc->resolution[a] > 0))
      return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: bad grid, padding or resolution");
    n3[a] = desc->grid[a] + 2 * desc->pad[a];
    if (!pow2_in(n3[a], 8, AXIS_MAX))
      return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: padded axis sizes must be powers of two in [8, 512]");
  }
  const bool avg = desc->absorbing[0] || desc->absorbing[1] || desc->absorbing[2];
  const bool zonly = desc->absorbing[2] && !desc->absorbing[0] && !desc->absorbing[1];
  if (avg && !zonly) return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: absorbing x or y boundaries are not supported");
  if (zonly && n3[2] > AXIS_MAX_AVG2)
    return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: padded z above 256 with an absorbing z boundary is not supported");
  const int prec = desc->precision;
  const bool c64 = prec != FM_PREC_F32;
  const int pwy = c64 ? pencils_per_warp<double>(n3[1]) : pencils_per_warp<float>(n3[1]);
  const int pwz = c64 ? pencils_per_warp<double>(zonly ? 2 * n3[2] : n3[2]) : pencils_per_warp<float>(zonly ? 2 * n3[2] : n3[2]);
  if (pwy <= 0 || pwz <= 0 || n3[0] % pwy || n3[0] % pwz)
    return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: x size too small for pencil tiling");
  const size_t esz = prec == FM_PREC_F64 ? 16 : 8;
  const char* xa = (const char*)x_dev;
  const char* ya = (const char*)y_dev;
  const size_t bytes = (size_t)nrhs * 3 * n3[0] * n3[1] * n3[2] * esz;
  if (xa < ya + bytes && ya < xa + bytes) return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: x and y overlap");
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return noalloc_fail(FM_ERR_CUDA, "cudaGetDevice failed");
  if (desc->device < 0 || desc->device >= FM_NOALLOC_MAX_DEVICES)
    return noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: device ordinal out of range");
  if (cudaSetDevice(desc->device) != cudaSuccess) return noalloc_fail(FM_ERR_CUDA, "cudaSetDevice failed");
  cudaStream_t st = (cudaStream_t)stream;
  fm_status s;
  if (prec == FM_PREC_F64) s = run<double, double>(*desc, k_bg, eps_imag, nrhs, x_dev, y_dev, st, desc->device);
  else if (prec == FM_PREC_F32_MATH64) s = run<float, double>(*desc, k_bg, eps_imag, nrhs, x_dev, y_dev, st, desc->device);
  else if (prec == FM_PREC_F32) s = run<float, float>(*desc, k_bg, eps_imag, nrhs, x_dev, y_dev, st, desc->device);
  else s = noalloc_fail(FM_ERR_INVALID, "fm_green_apply_noalloc: unknown precision");
  cudaSetDevice(prev);
  return s;
}
