"""CPU oracle for the convergent Born series (CBS) solve of FrequencyMaxwell.jl.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA library: only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import it.  The product path (``fmcuda`` + ``libfmcuda.so``) never calls it.

It restates, in numpy/scipy FP64 (or FP32 for emulation), the reference's
``solve(solver, source, medium)`` path.  Every function cites the reference file
and lines it follows (paths inside the FrequencyMaxwell.jl project).

Pinning.  The reference is Julia; Julia is not installed here, so the reference
cannot be run and its solve output is not available.  No reference test calls
``solve``, so **parity of the solve itself is unpinned** by the reference.  What
is pinned are the constants the reference tests assert (boundary-condition
padding/shift/flags, phantom voxel values and volume, plane-wave impedance,
polarisation orthogonality and superposition): ``tests/test_oracle_pins.py``
checks this module against each of them.  The oracle is further checked for
self-consistency (FFT Green apply vs a dense direct DFT, GMRES vs a dense
solve, GMRES vs BiCGStab vs Richardson agreement).

Third-party arithmetic that is not under the reference tree and is restated
from its published algorithm (versions unpinned: the reference commits no
Manifest):
  * Krylov.jl GMRES (Saad & Schultz 1986) as driven by LinearSolve.jl 2
    ``KrylovJL_GMRES`` (no restart, modified Gram-Schmidt, Givens rotations,
    left preconditioner applied with ``ldiv!``, warm start ``u0``, stop when
    the preconditioned residual estimate <= atol + rtol*||r0||).
  * Krylov.jl BiCGStab (van der Vorst 1992), shadow vector c = b.
  * FFTW: unnormalised forward DFT with exp(-i...), inverse normalised 1/N.
"""
from __future__ import annotations

import functools
import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np
import scipy.fft as sfft
import threadpoolctl

_WORKERS = os.cpu_count() or 1
_POOL: Optional[ThreadPoolExecutor] = None


def _slab_map(fn, nz: int) -> None:
    """Run ``fn(z_slice)`` over contiguous z slabs on a thread pool.

    The arithmetic per element is unchanged; numpy releases the GIL inside its loops, so
    the slabs run in parallel.  Arrays are Fortran-ordered (x fastest), so a z slab of a
    (nx, ny, nz[, 3]) array is a contiguous block (per component)."""
    global _POOL
    n = max(1, min(_WORKERS, nz))
    bounds = [nz * i // n for i in range(n + 1)]
    slabs = [slice(bounds[i], bounds[i + 1]) for i in range(n) if bounds[i + 1] > bounds[i]]
    if n == 1:
        fn(slabs[0])
        return
    if _POOL is None:
        _POOL = ThreadPoolExecutor(_WORKERS)
    for f in [_POOL.submit(fn, sl) for sl in slabs]:
        f.result()

# ----------------------------------------------------------------------------
# Boundary conditions  (src/solvers/boundary_conditions.jl)
# ----------------------------------------------------------------------------

TANH, EXPONENTIAL, TUKEY = "tanh", "exponential", "tukey"


@dataclass(frozen=True)
class PeriodicBC:
    """PeriodicBoundaryCondition (boundary_conditions.jl:157-181)."""


@dataclass(frozen=True)
class AbsorbingBC:
    """AbsorbingBoundaryCondition with its validation (boundary_conditions.jl:335-395)."""
    thickness: float
    attenuation_thickness: float
    sharpness: float = 0.9
    profile: str = TANH

    def __post_init__(self):
        if not self.thickness > 0:
            raise ValueError(f"thickness must be positive, got: {self.thickness}")
        if not self.attenuation_thickness > 0:
            raise ValueError("attenuation_thickness must be positive")
        if not self.attenuation_thickness <= self.thickness:
            raise ValueError("attenuation_thickness must be <= thickness")
        if not (0 <= self.sharpness <= 1):
            raise ValueError("sharpness must be in [0, 1]")
        if self.profile not in (TANH, EXPONENTIAL, TUKEY):
            raise ValueError(f"Unknown attenuation profile: {self.profile}")


def julia_round(x: float) -> int:
    """Julia ``round(Int, x)``: nearest, ties to even (Python's round does the same)."""
    return int(round(x))


def padding_pixels(bc, resolution: float) -> int:
    """boundary_conditions.jl:450-459."""
    if isinstance(bc, PeriodicBC):
        return 0
    return julia_round(bc.thickness / (resolution * 2))


def subpixel_shift(bc) -> float:
    """boundary_conditions.jl:518-527."""
    return 0.0 if isinstance(bc, PeriodicBC) else 0.25


def requires_padding(bc) -> bool:
    """boundary_conditions.jl:567-573."""
    return isinstance(bc, AbsorbingBC)


def requires_averaging(bc) -> bool:
    """boundary_conditions.jl:609-615."""
    return isinstance(bc, AbsorbingBC)


def attenuation_window(profile: str, L: int) -> np.ndarray:
    """boundary_conditions.jl:632-658.

    The Tanh form keeps the reference's operator order: (tanh(x)/tanh(2.5) - tanh(-2.5))/2,
    which spans about [-0.0067, 0.9933] rather than [0, 1].
    """
    if L <= 0:
        return np.zeros(0)
    if profile == TANH:
        v = np.tanh(np.linspace(-2.5, 2.5, L))
        return (v / math.tanh(2.5) - math.tanh(-2.5)) / 2
    x = np.linspace(0.0, 1.0, L)
    if profile == EXPONENTIAL:
        return np.exp(-(((1.0 - x) / 0.3) ** 2))
    if profile == TUKEY:
        return 0.5 * (1.0 + np.cos(np.pi * (1.0 - x)))
    raise ValueError(profile)


# ----------------------------------------------------------------------------
# Solver configuration  (src/solvers/convergent_born.jl:87-233, 250-260)
# ----------------------------------------------------------------------------

@dataclass
class SolverConfig:
    resolution: Tuple[float, float, float]
    grid_size: Tuple[int, int, int]
    boundary_conditions: Tuple[object, object, object]
    iterations_max: int = -1
    tolerance: float = 1e-6
    method: str = "gmres"            # "gmres" | "bicgstab" | "richardson"

    def __post_init__(self):
        # convergent_born.jl:117-121 and 207-217 (single BC -> all axes)
        if not isinstance(self.boundary_conditions, (tuple, list)):
            self.boundary_conditions = (self.boundary_conditions,) * 3
        self.boundary_conditions = tuple(self.boundary_conditions)
        self.resolution = tuple(float(r) for r in self.resolution)
        self.grid_size = tuple(int(n) for n in self.grid_size)
        if not all(r > 0 for r in self.resolution):
            raise ValueError("all resolution components must be positive")
        if not all(n > 0 for n in self.grid_size):
            raise ValueError("all grid_size components must be positive")
        if not (0 <= self.tolerance <= 1):
            raise ValueError("tolerance must be in [0, 1]")

    @property
    def padding(self) -> Tuple[int, int, int]:
        return tuple(padding_pixels(self.boundary_conditions[d], self.resolution[d]) for d in range(3))

    @property
    def padded_size(self) -> Tuple[int, int, int]:
        return tuple(self.grid_size[d] + 2 * self.padding[d] for d in range(3))

    @property
    def shifts(self) -> Tuple[float, float, float]:
        return tuple(subpixel_shift(bc) for bc in self.boundary_conditions)

    @property
    def use_averaging(self) -> bool:
        return any(requires_averaging(bc) for bc in self.boundary_conditions)

    def roi(self) -> Tuple[int, ...]:
        """compute_ROI, 1-based inclusive bounds (convergent_born.jl:250-260)."""
        p, g = self.padding, self.grid_size
        return (p[0] + 1, p[0] + g[0], p[1] + 1, p[1] + g[1], p[2] + 1, p[2] + g[2])

    def crop(self, f: np.ndarray) -> np.ndarray:
        """crop_to_ROI (convergent_born.jl:951-960; electromagnetic_field.jl:288-303)."""
        r = self.roi()
        return f[r[0] - 1:r[1], r[2] - 1:r[3], r[4] - 1:r[5], ...]


# ----------------------------------------------------------------------------
# Potential  (convergent_born.jl:619-675, 807-944)
# ----------------------------------------------------------------------------

@dataclass
class Potential:
    V: np.ndarray            # padded, attenuated, including the -i*eps_imag shift
    eps_imag: float
    k_bg: float
    Bornmax: int
    wavelength: float

    @property
    def k_square(self) -> complex:
        # convergent_born.jl:663
        return complex(self.k_bg ** 2, self.eps_imag)


def pad_zeros(arr: np.ndarray, pad: Sequence[int]) -> np.ndarray:
    """_pad_array with mode :replicate, which pads zeros (convergent_born.jl:807-858, stubs 865-883)."""
    if all(p == 0 for p in pad):
        return arr.copy()
    shp = tuple(arr.shape[d] + 2 * pad[d] for d in range(3)) + arr.shape[3:]
    out = np.zeros(shp, dtype=arr.dtype, order="F")
    out[pad[0]:pad[0] + arr.shape[0], pad[1]:pad[1] + arr.shape[1], pad[2]:pad[2] + arr.shape[2], ...] = arr
    return out


def attenuation_filters(cfg: SolverConfig) -> List[Optional[np.ndarray]]:
    """Per-axis 1-D filters of _apply_attenuation_to_potential! (convergent_born.jl:893-944)."""
    out: List[Optional[np.ndarray]] = []
    for d in range(3):
        bc = cfg.boundary_conditions[d]
        if not requires_padding(bc):
            out.append(None)
            continue
        max_L = padding_pixels(bc, cfg.resolution[d])
        att_px = julia_round(bc.attenuation_thickness / (cfg.resolution[d] * 2))
        L = min(max_L, att_px)
        if max_L == 0:
            out.append(None)
            continue
        w = attenuation_window(bc.profile, L)
        w = w * bc.sharpness + (1 - bc.sharpness)
        roi_size = cfg.grid_size[d]
        rem = max_L - L
        out.append(np.concatenate([w, np.ones(roi_size + 2 * rem), w[::-1]]))
    return out


def build_potential(cfg: SolverConfig, permittivity: np.ndarray, permittivity_bg: float,
                    wavelength: float, dtype=np.complex128) -> Potential:
    """_initialize_solver! (convergent_born.jl:619-675)."""
    perm = np.asarray(permittivity)
    if perm.shape != cfg.grid_size:
        raise ValueError("medium grid_size must match solver grid_size")
    k_bg = 2 * math.pi * math.sqrt(permittivity_bg) / wavelength          # :630
    V0 = (k_bg ** 2 * (perm / permittivity_bg - 1)).astype(np.complex128)  # :631-632
    V = pad_zeros(np.asfortranarray(V0), cfg.padding)                     # :635-638
    eps_imag = max(2.0 ** -20, float(np.max(np.abs(V))) * 1.01)            # :641
    V = V - 1j * eps_imag                                                  # :644
    for d, f in enumerate(attenuation_filters(cfg)):                       # :647
        if f is None:
            continue
        shp = [1, 1, 1]
        shp[d] = -1
        V = V * f.reshape(shp)
    if cfg.iterations_max < 0:                                             # :653-660
        steps = abs(2 * k_bg / eps_imag)
        extent = float(np.linalg.norm(np.array(cfg.padded_size) * np.array(cfg.resolution)))
        born_opt = math.ceil(extent / steps / 2 + 1) * 2
        Bornmax = born_opt * abs(cfg.iterations_max)
    else:
        Bornmax = cfg.iterations_max
    return Potential(np.asfortranarray(V.astype(dtype)), eps_imag, k_bg, Bornmax, wavelength)


# ----------------------------------------------------------------------------
# Dyadic Green convolution  (src/core/dyadic_green.jl)
# ----------------------------------------------------------------------------

def green_k_index(n: int) -> np.ndarray:
    """rem(i + floor(N/2) - 1, N) - floor(N/2) for i = 1..N (dyadic_green.jl:203-208)."""
    i = np.arange(1, n + 1)
    h = n // 2
    return np.remainder(i + h - 1, n) - h


def curl_k_index(n: int) -> np.ndarray:
    """i <= N÷2 ? i-1 : i-N-1 for i = 1..N (curl.jl:84-86); differs from the Green index for odd N."""
    i = np.arange(1, n + 1)
    return np.where(i <= n // 2, i - 1, i - n - 1)


def _fft3(a):
    """Unnormalised 3-D DFT over the spatial axes (FFTW's forward ``fft``).  The transform runs on
    the transposed (C-ordered) view so a Fortran-ordered input gives a Fortran-ordered output."""
    nd = a.ndim
    return sfft.fftn(a.T, axes=tuple(range(nd - 3, nd)), workers=_WORKERS).T


def _ifft3(a):
    """1/N-normalised inverse 3-D DFT over the spatial axes (FFTW's ``ifft``)."""
    nd = a.ndim
    return sfft.ifftn(a.T, axes=tuple(range(nd - 3, nd)), workers=_WORKERS).T


def phase_ramp(shape3, shifts, reverse: bool, dtype=np.complex128) -> np.ndarray:
    """multiply_phase_ramp_kernel! factor exp(-/+ 2*pi*i*sum_d (idx_d-1)*s_d/N_d) (dyadic_green.jl:243-266)."""
    return _phase_ramp_cached(tuple(int(n) for n in shape3), tuple(float(s) for s in shifts), bool(reverse),
                              np.dtype(dtype).str).copy(order="F")


@functools.lru_cache(maxsize=16)
def _phase_ramp_cached(shape3, shifts, reverse, dtype_str) -> np.ndarray:
    dtype = np.dtype(dtype_str)
    ph = np.zeros(shape3)
    for d in range(3):
        if shifts[d] == 0:
            continue
        idx = np.arange(shape3[d]) * shifts[d] / shape3[d]
        shp = [1, 1, 1]
        shp[d] = -1
        ph = ph + idx.reshape(shp)
    sgn = 1.0 if reverse else -1.0
    out = np.asfortranarray(np.exp(sgn * 2j * np.pi * ph).astype(dtype))
    out.flags.writeable = False
    return out


def _green_axes(shape3, freq_res, shifts, rdt):
    kx = (freq_res[0] * (green_k_index(shape3[0]) + shifts[0])).astype(rdt).reshape(-1, 1, 1)
    ky = (freq_res[1] * (green_k_index(shape3[1]) + shifts[1])).astype(rdt).reshape(1, -1, 1)
    kz = (freq_res[2] * (green_k_index(shape3[2]) + shifts[2])).astype(rdt).reshape(1, 1, -1)
    return kx, ky, kz


def _green_multiply_into(src_hat: np.ndarray, out: np.ndarray, freq_res, shifts, k_square: complex) -> None:
    """out <- Green(src_hat); ``out`` may be ``src_hat`` itself.  Same arithmetic as green_multiply."""
    rdt = np.float64 if src_hat.dtype == np.complex128 else np.float32
    kx, ky, kz = _green_axes(src_hat.shape[:3], freq_res, shifts, rdt)
    ksq = src_hat.dtype.type(k_square)

    def slab(sl):
        kzs = kz[:, :, sl]
        s1, s2, s3 = src_hat[:, :, sl, 0], src_hat[:, :, sl, 1], src_hat[:, :, sl, 2]
        kE = (kx * s1 + ky * s2 + kzs * s3) / ksq
        D = np.abs(kx * kx + ky * ky + kzs * kzs) - ksq
        o1 = (s1 - kx * kE) / D
        o2 = (s2 - ky * kE) / D
        o3 = (s3 - kzs * kE) / D
        out[:, :, sl, 0] = o1
        out[:, :, sl, 1] = o2
        out[:, :, sl, 2] = o3

    _slab_map(slab, src_hat.shape[2])


def green_multiply(src_hat: np.ndarray, freq_res, shifts, k_square: complex) -> np.ndarray:
    """multiply_Green_kernel! (dyadic_green.jl:189-221).  k.E is divided by the complex k_square:
    kE = (k . E)/k_sq, D = |k|^2 - k_sq, E_c <- (E_c - k_c kE)/D."""
    out = np.empty(src_hat.shape, dtype=src_hat.dtype, order="F")
    _green_multiply_into(src_hat, out, freq_res, shifts, k_square)
    return out


def single_convolution(src: np.ndarray, cfg: SolverConfig, k_square: complex, shifts) -> np.ndarray:
    """_apply_single_convolution! (dyadic_green.jl:161-179): ramp(-), FFT, Green, IFFT, ramp(+)."""
    shape3 = src.shape[:3]
    freq_res = [2 * math.pi / (shape3[d] * cfg.resolution[d]) for d in range(3)]
    dt = src.dtype
    shifted = any(s != 0 for s in shifts)
    x = np.empty(src.shape, dtype=dt, order="F")
    if shifted:
        rf = _phase_ramp_cached(tuple(shape3), tuple(float(s) for s in shifts), False, np.dtype(dt).str)

        def pre(sl):
            for c in range(3):
                np.multiply(src[:, :, sl, c], rf[:, :, sl], out=x[:, :, sl, c])
        _slab_map(pre, shape3[2])
    else:
        x[...] = src
    x = _fft3(x)
    if x.dtype != dt:
        x = x.astype(dt, order="F")
    _green_multiply_into(x, x, freq_res, shifts, k_square)
    x = _ifft3(x)
    if x.dtype != dt:
        x = x.astype(dt, order="F")
    if shifted:
        rr = _phase_ramp_cached(tuple(shape3), tuple(float(s) for s in shifts), True, np.dtype(dt).str)

        def post(sl):
            for c in range(3):
                np.multiply(x[:, :, sl, c], rr[:, :, sl], out=x[:, :, sl, c])
        _slab_map(post, shape3[2])
    return x


def green_conv(src: np.ndarray, cfg: SolverConfig, k_square: complex) -> np.ndarray:
    """conv!(::DyadicGreen, src) with the (G(+s) + G(-s))/2 average (dyadic_green.jl:127-152)."""
    shifts = cfg.shifts
    src = np.asfortranarray(src)
    if not cfg.use_averaging:
        return single_convolution(src, cfg, k_square, shifts)
    a = single_convolution(src, cfg, k_square, shifts)
    b = single_convolution(src, cfg, k_square, tuple(-s for s in shifts))

    def avg(sl):
        a[:, :, sl] += b[:, :, sl]
        a[:, :, sl] /= 2
    _slab_map(avg, a.shape[2])
    return a


def _times_V(V: np.ndarray, x: np.ndarray, scale=None) -> np.ndarray:
    """V .* x per component (times a scalar ``scale`` after the product when given)."""
    x = np.asfortranarray(x)
    out = np.empty(x.shape, dtype=np.result_type(V.dtype, x.dtype), order="F")

    def slab(sl):
        for c in range(3):
            o = out[:, :, sl, c]
            np.multiply(V[:, :, sl], x[:, :, sl, c], out=o)
            if scale is not None:
                o *= scale
    _slab_map(slab, x.shape[2])
    return out


def cbs_operator(x: np.ndarray, V: np.ndarray, cfg: SolverConfig, k_square: complex,
                 alpha=1.0, beta=0.0, y: Optional[np.ndarray] = None) -> np.ndarray:
    """CBSLinearOperator: y = beta*y + alpha*(x - G_avg(V.*x)) (convergent_born.jl:482-508)."""
    x = np.asfortranarray(x)
    psi = green_conv(_times_V(V, x), cfg, k_square)

    def slab(sl):
        r = x[:, :, sl] - psi[:, :, sl]
        if y is None or beta == 0:
            psi[:, :, sl] = alpha * r if alpha != 1.0 else r
        else:
            psi[:, :, sl] = beta * y[:, :, sl] + alpha * r
    _slab_map(slab, x.shape[2])
    return psi


def cbs_preconditioner(x: np.ndarray, V: np.ndarray, eps_imag: float) -> np.ndarray:
    """CBSPreconditioner ldiv!: y = (i/eps_imag) .* V .* x (convergent_born.jl:398-431)."""
    return _times_V(V, x, 1j / eps_imag)


# ----------------------------------------------------------------------------
# Krylov solvers (restated from Krylov.jl's published algorithms)
# ----------------------------------------------------------------------------

@dataclass
class KrylovResult:
    x: np.ndarray
    iters: int
    solved: bool
    residuals: List[float] = field(default_factory=list)


def _chunks(n: int):
    k = max(1, min(_WORKERS, n // 65536))
    b = [n * i // k for i in range(k + 1)]
    return [slice(b[i], b[i + 1]) for i in range(k)]


def _pool_map(fn, items):
    global _POOL
    if len(items) == 1:
        return [fn(items[0])]
    if _POOL is None:
        _POOL = ThreadPoolExecutor(_WORKERS)
    return [f.result() for f in [_POOL.submit(fn, it) for it in items]]


def _dot(a, b) -> complex:
    """Julia dot(a, b) = sum(conj(a) .* b), accumulated in complex128 (chunk partial sums added in
    chunk order)."""
    a = a.astype(np.complex128, copy=False)
    b = b.astype(np.complex128, copy=False)
    if a.strides != b.strides or not a.flags.f_contiguous:
        a, b = np.asfortranarray(a), np.asfortranarray(b)
    ar, br = a.ravel(order="K"), b.ravel(order="K")
    parts = _pool_map(lambda sl: complex(np.vdot(ar[sl], br[sl])), _chunks(ar.size))
    tot = 0j
    for p in parts:
        tot += p
    return tot


def _nrm(a) -> float:
    return float(np.sqrt(np.real(_dot(a, a))))


_BLK = 1 << 17


def _axpy_block(a, xs, ys, tmp) -> None:
    """ys <- ys + a*xs on one block (numpy loops release the GIL, so blocks run in parallel)."""
    t = tmp[:ys.size]
    np.multiply(xs, a, out=t)
    np.add(ys, t, out=ys)


def _axpy_dot(a: complex, xv: np.ndarray, yv: np.ndarray, zv: np.ndarray) -> complex:
    """One fused modified Gram-Schmidt stage: yv <- yv + a*xv, then return dot(zv, yv).

    Per element the arithmetic is that of the two separate steps; the pass runs in cache-sized
    blocks so yv is read once for both.  All three arrays are complex128 with equal strides."""
    xr, yr, zr = xv.ravel(order="K"), yv.ravel(order="K"), zv.ravel(order="K")
    a = complex(a)

    def part(sl):
        tmp = np.empty(_BLK, dtype=np.complex128)
        tot = 0j
        for s0 in range(sl.start, sl.stop, _BLK):
            b = slice(s0, min(s0 + _BLK, sl.stop))
            _axpy_block(a, xr[b], yr[b], tmp)
            tot += complex(np.vdot(zr[b], yr[b]))
        return tot
    parts = _pool_map(part, _chunks(yr.size))
    tot = 0j
    for p in parts:
        tot += p
    return tot


def _axpy(a: complex, xv: np.ndarray, yv: np.ndarray) -> None:
    """yv <- yv + a*xv in place."""
    if (yv.dtype == xv.dtype and yv.shape == xv.shape and yv.strides == xv.strides
            and (yv.flags.f_contiguous or yv.flags.c_contiguous)):
        xr, yr = xv.ravel(order="K"), yv.ravel(order="K")
        av = yv.dtype.type(a)

        def part(sl):
            tmp = np.empty(_BLK, dtype=yv.dtype)
            for s0 in range(sl.start, sl.stop, _BLK):
                b = slice(s0, min(s0 + _BLK, sl.stop))
                _axpy_block(av, xr[b], yr[b], tmp)
        _pool_map(part, _chunks(yr.size))
        return
    yv += yv.dtype.type(a) * xv


def sym_givens(a: complex, b: float):
    """Givens reflection with real c and complex s: [c s; conj(s) -c][a; b] = [rho; 0]."""
    abs_a = abs(a)
    if b == 0:
        return 1.0, 0j, a
    if abs_a == 0:
        return 0.0, 1 + 0j, complex(b)
    r = math.hypot(abs_a, b)
    c = abs_a / r
    s = (a / abs_a) * b / r
    rho = (a / abs_a) * r
    return c, s, rho


def gmres(apply_A, apply_M, b: np.ndarray, x0: np.ndarray, atol: float, rtol: float,
          itmax: int, restart: int = 0, callback=None) -> KrylovResult:
    """Left-preconditioned GMRES of Krylov.jl (see ``_gmres_impl``).  ``callback(k)``, when given,
    is called after inner iteration k (1-based, counted over restarts)."""
    with threadpoolctl.threadpool_limits(1, user_api="blas"):
        return _gmres_impl(apply_A, apply_M, b, x0, atol, rtol, itmax, restart, callback)


def bicgstab(apply_A, apply_M, b: np.ndarray, x0: np.ndarray, atol: float, rtol: float,
             itmax: int) -> KrylovResult:
    """Left-preconditioned BiCGStab of Krylov.jl (see ``_bicgstab_impl``)."""
    with threadpoolctl.threadpool_limits(1, user_api="blas"):
        return _bicgstab_impl(apply_A, apply_M, b, x0, atol, rtol, itmax)


def richardson(apply_A, apply_M, b: np.ndarray, x0: np.ndarray, atol: float, rtol: float,
               itmax: int) -> KrylovResult:
    """The plain convergent Born series (see ``_richardson_impl``)."""
    with threadpoolctl.threadpool_limits(1, user_api="blas"):
        return _richardson_impl(apply_A, apply_M, b, x0, atol, rtol, itmax)


def _gmres_impl(apply_A, apply_M, b: np.ndarray, x0: np.ndarray, atol: float, rtol: float,
                itmax: int, restart: int = 0, callback=None) -> KrylovResult:
    """Left-preconditioned GMRES with warm start, as Krylov.jl ``gmres`` runs it under LinearSolve
    (``KrylovJL_GMRES``: ``restart=false`` -> full GMRES whose basis grows; MGS; Givens).

    ``restart > 0`` gives GMRES(m) (restart every m inner iterations, x kept).
    Residual = M^{-1}(b - A x); stop when its estimate <= atol + rtol*||r0||.
    """
    x = np.asfortranarray(x0).copy(order="F")
    r0 = apply_M(b - apply_A(x))
    beta = _nrm(r0)
    rnorms = [beta]
    if beta == 0:
        return KrylovResult(x, 0, True, rnorms)
    eps = atol + rtol * beta
    btol = np.finfo(np.float64).eps ** 0.75
    it = 0
    solved = beta <= eps
    while not solved and it < itmax:
        if restart and it > 0:
            r0 = apply_M(b - apply_A(x))
        beta_p = _nrm(r0)
        Vb = [r0 / beta_p]
        z = [complex(beta_p)]
        cs, ss, H = [], [], []          # H[k] = column k of R (after rotations)
        inner = 0
        breakdown = False
        m = restart if restart else itmax - it
        while True:
            inner += 1
            q = apply_M(apply_A(Vb[-1]))
            col = []
            q = np.asfortranarray(q)
            fused = q.dtype == np.complex128 and all(v.strides == q.strides and v.dtype == q.dtype for v in Vb)
            for i in range(inner):
                # modified Gram-Schmidt: h_i = <v_i, q>; q <- q - h_i v_i (the update of stage i-1 and
                # the dot of stage i share one pass over q when the layouts allow it)
                if i == 0 or not fused:
                    h = _dot(Vb[i], q)
                else:
                    h = _axpy_dot(-col[-1], Vb[i - 1], q, Vb[i])
                col.append(h)
                if not fused:
                    _axpy(-h, Vb[i], q)
            if fused:
                _axpy(-col[-1], Vb[inner - 1], q)
            hb = _nrm(q)
            for i in range(inner - 1):
                t = cs[i] * col[i] + ss[i] * col[i + 1]
                col[i + 1] = np.conj(ss[i]) * col[i] - cs[i] * col[i + 1]
                col[i] = t
            c, s, rho = sym_givens(col[inner - 1], hb)
            col[inner - 1] = rho
            cs.append(c)
            ss.append(s)
            H.append(col)
            zk1 = np.conj(s) * z[inner - 1]
            z[inner - 1] = c * z[inner - 1]
            rnorm = abs(zk1)
            rnorms.append(rnorm)
            if callback is not None:
                callback(it + inner)
            solved = rnorm <= eps or (rnorm + 1.0 <= 1.0)
            breakdown = hb <= btol
            tired = (it + inner) >= itmax or inner >= m
            if solved or tired or breakdown:
                break
            Vb.append(q / hb)
            z.append(zk1)
        # back substitution R y = z
        y = list(z[:inner])
        for i in range(inner - 1, -1, -1):
            for j in range(inner - 1, i, -1):
                y[i] = y[i] - H[j][i] * y[j]
            if abs(H[i][i]) <= btol:
                y[: i + 1] = [0j] * (i + 1)
                break
            y[i] = y[i] / H[i][i]
        x = np.asfortranarray(x)
        for i in range(inner):
            _axpy(y[i], Vb[i], x)
        it += inner
        if breakdown:
            break
    return KrylovResult(x, it, bool(solved), rnorms)


def _bicgstab_impl(apply_A, apply_M, b: np.ndarray, x0: np.ndarray, atol: float, rtol: float,
                   itmax: int) -> KrylovResult:
    """Left-preconditioned BiCGStab (van der Vorst 1992) in the form of Krylov.jl ``bicgstab``:
    warm start solves A dx = b - A x0, shadow vector c = b, residual r = M^{-1}(b - A x)."""
    r0 = b - apply_A(x0)
    r = apply_M(r0)
    c = b
    p = r.copy()
    v = np.zeros_like(r)
    dx = np.zeros_like(r)
    rnorm = _nrm(r)
    rnorms = [rnorm]
    if rnorm == 0:
        return KrylovResult(x0.copy(), 0, True, rnorms)
    eps = atol + rtol * rnorm
    next_rho = _dot(c, r)
    if next_rho == 0:
        return KrylovResult(x0.copy(), 0, False, rnorms)
    solved = rnorm <= eps
    it = 0
    while not solved and it < itmax:
        it += 1
        rho = next_rho
        v = apply_M(apply_A(p))
        alpha = rho / _dot(c, v)
        s = r - alpha * v
        dx = dx + alpha * p
        t = apply_M(apply_A(s))
        omega = _dot(t, s) / _dot(t, t)
        dx = dx + omega * s
        r = s - omega * t
        next_rho = _dot(c, r)
        beta = (next_rho / rho) * (alpha / omega)
        p = r + beta * (p - omega * v)
        rnorm = _nrm(r)
        rnorms.append(rnorm)
        solved = rnorm <= eps or (rnorm + 1.0 <= 1.0)
        if alpha == 0 or np.isnan(alpha):
            break
    return KrylovResult(x0 + dx, it, bool(solved), rnorms)


def _richardson_impl(apply_A, apply_M, b: np.ndarray, x0: np.ndarray, atol: float, rtol: float,
                     itmax: int) -> KrylovResult:
    """Plain convergent Born series: x <- x + M^{-1}(b - A x), with the same stopping rule as the
    Krylov forms (||M^{-1}(b - A x)|| <= atol + rtol*||M^{-1}(b - A x0)||)."""
    x = x0.copy()
    r = apply_M(b - apply_A(x))
    r0n = _nrm(r)
    rnorms = [r0n]
    eps = atol + rtol * r0n
    it = 0
    solved = r0n <= eps
    while not solved and it < itmax:
        x = x + r
        it += 1
        r = apply_M(b - apply_A(x))
        rn = _nrm(r)
        rnorms.append(rn)
        solved = rn <= eps
    return KrylovResult(x, it, bool(solved), rnorms)


# ----------------------------------------------------------------------------
# Curl / magnetic field  (src/core/curl.jl; convergent_born.jl:784-800)
# ----------------------------------------------------------------------------

def curl(E: np.ndarray, resolution) -> np.ndarray:
    """conv(::Curl, E): ifft(ik x fft(E)) with the curl k-index (curl.jl:55-116)."""
    shape3 = E.shape[:3]
    fr = [2 * math.pi / (shape3[d] * resolution[d]) for d in range(3)]
    dt = E.dtype
    kx = (fr[0] * curl_k_index(shape3[0])).reshape(-1, 1, 1)
    ky = (fr[1] * curl_k_index(shape3[1])).reshape(1, -1, 1)
    kz = (fr[2] * curl_k_index(shape3[2])).reshape(1, 1, -1)
    F = _fft3(E).astype(dt)
    s1, s2, s3 = F[..., 0], F[..., 1], F[..., 2]
    out = np.empty_like(F)
    out[..., 0] = 1j * ky * s3 - 1j * kz * s2
    out[..., 1] = 1j * kz * s1 - 1j * kx * s3
    out[..., 2] = 1j * kx * s2 - 1j * ky * s1
    return _ifft3(out).astype(dt)


def magnetic_field(E: np.ndarray, resolution, wavelength: float) -> np.ndarray:
    """_compute_magnetic_field: H = -i*lambda/(2*pi*377) * curl(E) (convergent_born.jl:784-800)."""
    return (-1j * wavelength / (2 * math.pi * 377)) * curl(E, resolution)


# ----------------------------------------------------------------------------
# Plane-wave sources  (src/sources/plane_wave.jl; src/sources/field_generation.jl)
# ----------------------------------------------------------------------------

@dataclass
class PlaneWave:
    """PlaneWaveSource with its validation (plane_wave.jl:63-116)."""
    wavelength: float
    polarization: Sequence[complex]
    k_vector: Sequence[float]
    amplitude: float = 1.0
    phase: float = 0.0

    def __post_init__(self):
        self.polarization = np.asarray(self.polarization, dtype=np.complex128)
        self.k_vector = np.asarray(self.k_vector, dtype=np.float64)
        if not self.wavelength > 0:
            raise ValueError("wavelength must be positive")
        if not self.amplitude >= 0:
            raise ValueError("amplitude must be non-negative")
        if not abs(np.linalg.norm(self.k_vector) - 1) < 1e-10:
            raise ValueError("k_vector must be normalized (|k| = 1)")
        if not abs(np.real(np.vdot(self.polarization, self.k_vector))) < 1e-10:
            raise ValueError("polarization must be transverse to k_vector")


def source_wavelength(sources) -> float:
    """plane_wave.jl:125-141 (exact equality across a vector of sources)."""
    if isinstance(sources, PlaneWave):
        return sources.wavelength
    w = sources[0].wavelength
    for s in sources[1:]:
        if s.wavelength != w:
            raise ValueError("All sources must have the same wavelength for coherent superposition")
    return w


def plane_wave_polarisations(src: PlaneWave, permittivity_bg: float):
    """E_perp, H_perp and k_vec of generate_incident_field (plane_wave.jl:218-232)."""
    k0 = 2 * math.pi / src.wavelength
    k_bg = k0 * math.sqrt(permittivity_bg)
    k_hat = src.k_vector / np.linalg.norm(src.k_vector)
    k_vec = k_bg * k_hat
    E0 = src.polarization / np.linalg.norm(src.polarization)
    E_perp = E0 - np.vdot(E0, k_hat) * k_hat          # Julia dot conjugates its first argument
    E_perp = E_perp / np.linalg.norm(E_perp)
    H_perp = np.cross(k_hat, E_perp) / (377 / math.sqrt(permittivity_bg))
    return E_perp, H_perp, k_vec


def incident_field_single(src: PlaneWave, cfg: SolverConfig, permittivity_bg: float = 1.0,
                          dtype=np.complex128):
    """generate_incident_field(::PlaneWaveSource) on the padded grid (plane_wave.jl:198-268)."""
    pad, g, res = cfg.padding, cfg.grid_size, cfg.resolution
    P = cfg.padded_size
    E_perp, H_perp, k_vec = plane_wave_polarisations(src, permittivity_bg)
    center = [(g[d] - 1) * res[d] / 2 for d in range(3)]
    r = [(np.arange(P[d]) - pad[d]) * res[d] - center[d] for d in range(3)]
    phase = (k_vec[0] * r[0]).reshape(-1, 1, 1) + (k_vec[1] * r[1]).reshape(1, -1, 1) \
        + (k_vec[2] * r[2]).reshape(1, 1, -1) + src.phase
    amp = src.amplitude * np.exp(1j * phase)
    E = np.empty(P + (3,), dtype=np.complex128, order="F")
    H = np.empty(P + (3,), dtype=np.complex128, order="F")
    for c in range(3):
        E[..., c] = amp * E_perp[c]
        H[..., c] = amp * H_perp[c]
    return E.astype(dtype), H.astype(dtype)


def incident_field(sources, cfg: SolverConfig, permittivity_bg: float = 1.0, dtype=np.complex128):
    """Coherent sum over sources (field_generation.jl:42-78)."""
    if isinstance(sources, PlaneWave):
        return incident_field_single(sources, cfg, permittivity_bg, dtype)
    if len(sources) == 0:
        raise ValueError("sources vector cannot be empty")
    w0 = sources[0].wavelength
    for s in sources[1:]:
        if not math.isclose(s.wavelength, w0, rel_tol=1e-10):
            raise ValueError("All sources must have the same wavelength for coherent interference.")
    E, H = incident_field_single(sources[0], cfg, permittivity_bg, dtype)
    for s in sources[1:]:
        e, h = incident_field_single(s, cfg, permittivity_bg, dtype)
        E = E + e
        H = H + h
    return E, H


# ----------------------------------------------------------------------------
# Phantoms  (src/medium/phantoms.jl)
# ----------------------------------------------------------------------------

def fill_sphere(ph: np.ndarray, center, radius: float, value: complex) -> None:
    """_fill_sphere! (phantoms.jl:212-247); centre in 1-based voxel coordinates, <= r^2, bbox by round."""
    g = ph.shape
    r2 = radius ** 2
    lo = [max(1, julia_round(center[d] - radius)) for d in range(3)]
    hi = [min(g[d], julia_round(center[d] + radius)) for d in range(3)]
    if any(hi[d] < lo[d] for d in range(3)):
        return
    ii = np.arange(lo[0], hi[0] + 1).reshape(-1, 1, 1)
    jj = np.arange(lo[1], hi[1] + 1).reshape(1, -1, 1)
    kk = np.arange(lo[2], hi[2] + 1).reshape(1, 1, -1)
    d2 = (ii - center[0]) ** 2 + (jj - center[1]) ** 2 + (kk - center[2]) ** 2
    sub = ph[lo[0] - 1:hi[0], lo[1] - 1:hi[1], lo[2] - 1:hi[2]]
    sub[d2 <= r2] = value


def phantom_bead(grid_size, permittivity_profile, pixel_radius: float, permittivity_bg: float = 1.0,
                 bead_distance: Optional[float] = None) -> np.ndarray:
    """phantom_bead (phantoms.jl:58-106): beads stacked along z about the grid centre (N+1)/2."""
    if bead_distance is None:
        bead_distance = 2 * pixel_radius
    if not all(n > 0 for n in grid_size):
        raise ValueError("grid_size must have positive dimensions")
    if not pixel_radius > 0:
        raise ValueError("pixel_radius must be positive")
    if len(permittivity_profile) == 0:
        raise ValueError("permittivity_profile cannot be empty")
    if not permittivity_bg > 0:
        raise ValueError("permittivity_bg must be positive")
    ph = np.full(tuple(grid_size), complex(permittivity_bg), dtype=np.complex128, order="F")
    num = len(permittivity_profile)
    c = [(grid_size[d] + 1) / 2 for d in range(3)]
    for b in range(1, num + 1):
        zoff = (b - (num + 1) / 2) * bead_distance
        bc = (c[0], c[1], c[2] + zoff)
        if bc[2] < 1 or bc[2] > grid_size[2]:
            continue
        val = complex(permittivity_profile[(b - 1) % num])
        fill_sphere(ph, bc, pixel_radius, val)
    return ph


def phantom_plate(grid_size, permittivity_profile, thickness_pixel: float, permittivity_bg: float = 1.0,
                  plate_normal: int = 3) -> np.ndarray:
    """phantom_plate (phantoms.jl:156-199)."""
    ph = np.full(tuple(grid_size), complex(permittivity_bg), dtype=np.complex128, order="F")
    cpos = (grid_size[plate_normal - 1] + 1) / 2
    half = thickness_pixel / 2
    s = max(1, julia_round(cpos - half))
    e = min(grid_size[plate_normal - 1], julia_round(cpos + half))
    sl = [slice(None)] * 3
    sl[plate_normal - 1] = slice(s - 1, e)
    ph[tuple(sl)] = complex(permittivity_profile[0])
    return ph


def fill_cylinder(ph: np.ndarray, center, radius: float, axis_start: int, axis_end: int, axis: int,
                  value: complex) -> None:
    """_fill_cylinder! (phantoms.jl:315-362): along `axis` (1..3) from axis_start to axis_end (1-based,
    inclusive), the voxels whose squared distance over the two other axes (in increasing axis order) is <= r^2."""
    g = ph.shape
    r2 = radius ** 2
    a = axis - 1
    o = [d for d in range(3) if d != a]
    u = np.arange(1, g[o[0]] + 1).reshape(-1, 1) - center[o[0]]
    v = np.arange(1, g[o[1]] + 1).reshape(1, -1) - center[o[1]]
    disk = u * u + v * v <= r2
    for idx in range(axis_start - 1, axis_end):
        sl = [slice(None)] * 3
        sl[a] = idx
        ph[tuple(sl)][disk] = value


def phantom_cylinder(grid_size, permittivity_profile, radius_pixel: float, permittivity_bg: float = 1.0,
                     height_pixel: Optional[float] = None, axis: int = 3) -> np.ndarray:
    """phantom_cylinder (phantoms.jl:272-313): a cylinder about the grid centre (N+1)/2 along `axis`, extent
    [max(1, round(c - h/2)), min(N, round(c + h/2))]."""
    if height_pixel is None:
        height_pixel = 2 * radius_pixel
    ph = np.full(tuple(grid_size), complex(permittivity_bg), dtype=np.complex128, order="F")
    c = [(grid_size[d] + 1) / 2 for d in range(3)]
    s = max(1, julia_round(c[axis - 1] - height_pixel / 2))
    e = min(grid_size[axis - 1], julia_round(c[axis - 1] + height_pixel / 2))
    fill_cylinder(ph, c, radius_pixel, s, e, axis, complex(permittivity_profile[0]))
    return ph


# ----------------------------------------------------------------------------
# solve  (convergent_born.jl:565-600, 703-774)
# ----------------------------------------------------------------------------

@dataclass
class SolveResult:
    E: np.ndarray             # total field, cropped to the ROI, (Nx, Ny, Nz, 3)
    H: np.ndarray
    E_scat_padded: np.ndarray
    iterations: int
    residual: float
    solved: bool
    potential: Potential
    residuals: List[float] = field(default_factory=list)


def solve(cfg: SolverConfig, sources, permittivity: np.ndarray, permittivity_bg: float,
          dtype=np.complex128, method: Optional[str] = None, restart: int = 0,
          atol: Optional[float] = None, rtol: Optional[float] = None,
          itmax: Optional[int] = None, callback=None) -> SolveResult:
    """LinearSolve.solve(::ConvergentBornSolver, sources, medium) (convergent_born.jl:565-600).

    ``callback(k)`` is passed to GMRES (called after each iteration k)."""
    method = method or cfg.method
    wl = source_wavelength(sources)
    pot = build_potential(cfg, permittivity, permittivity_bg, wl, dtype)
    E_inc, H_inc = incident_field(sources, cfg, permittivity_bg, dtype)
    V = pot.V
    S = V[..., None] * E_inc + (1j * pot.eps_imag) * E_inc                 # :585-586
    if pot.Bornmax < 1:
        raise RuntimeError("Bornmax < 1: the reference leaves the field undefined")
    ksq = pot.k_square
    b = green_conv(S.astype(dtype), cfg, ksq)                               # :720-728
    x0 = b.copy(order="F")
    A = lambda v: cbs_operator(v, V, cfg, ksq)
    M = lambda v: cbs_preconditioner(v, V, pot.eps_imag).astype(dtype, copy=False)
    rt = cfg.tolerance if rtol is None else rtol
    at = cfg.tolerance * 1e-2 if atol is None else atol                    # :743-747
    mi = max(pot.Bornmax * 2, 100) if itmax is None else itmax
    if method == "gmres":
        res = gmres(A, M, b, x0, at, rt, mi, restart, callback)
    elif method == "bicgstab":
        res = bicgstab(A, M, b, x0, at, rt, mi)
    elif method == "richardson":
        res = richardson(A, M, b, x0, at, rt, mi)
    else:
        raise ValueError(method)
    Es = res.x.astype(dtype)
    Hs = magnetic_field(Es, cfg.resolution, wl).astype(dtype)              # :770
    E = cfg.crop(Es + E_inc)                                                # :596-597
    H = cfg.crop(Hs + H_inc)
    return SolveResult(E, H, Es, res.iters, res.residuals[-1], res.solved, pot, res.residuals)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b||_2 / ||b||_2 in FP64."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
