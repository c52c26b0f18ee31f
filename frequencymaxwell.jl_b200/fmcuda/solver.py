"""ConvergentBornSolver and solve (mirror of src/solvers/convergent_born.jl) on libfmcuda.

``solve(solver, sources, medium)`` keeps the reference's signature and
semantics: sources may be one PlaneWaveSource or a list summed coherently; the
result is the total field cropped to the region of interest; non-convergence
warns and still returns the field; ``solver.iteration_count`` and
``solver.residual_history`` are filled as in convergent_born.jl:761-766.

All numerics run on the GPU through the C ABI; the host only computes the 1-D
attenuation windows and packs parameters.  ``solve_batch`` is new: it runs many
independent right-hand sides (illuminations) of one medium in one batched solve.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L
from .boundary import (AbsorbingBoundaryCondition, AbstractBoundaryCondition, PeriodicBoundaryCondition,
                       attenuation_filter, padding_pixels, requires_averaging, requires_padding, subpixel_shift)
from .fields import ElectromagneticField
from .medium import DevicePhantom, Medium, grid_size as medium_grid_size
from .sources import PlaneWaveSource, as_list, source_wavelength


# ---- linear-solver selectors (the reference passes LinearSolve.jl algorithm objects) ----
@dataclass(frozen=True)
class KrylovJL_GMRES:
    """GMRES as LinearSolve's KrylovJL_GMRES runs it (default: no restart).  ``gmres_restart`` > 0
    gives GMRES(m).  ``ortho`` picks the Gram-Schmidt variant ("mgs" as Krylov.jl, "cgs", "cgs2", or "block":
    s-step GMRES with ``block_size`` vectors per block, full GMRES only; ``block_vectors`` "fp64" keeps the raw
    block vectors in complex FP64 on plans that compute in FP64, "storage" in the plan's storage type,
    "fp64-ortho" as "fp64" and stores each block orthonormalised);
    None chooses MGS for FP64 (Krylov.jl's choice) and classical Gram-Schmidt for the FP32 forms."""
    gmres_restart: int = 0
    ortho: Optional[str] = None
    block_size: int = 8
    block_vectors: str = "fp64-ortho"


@dataclass(frozen=True)
class KrylovJL_BICGSTAB:
    """BiCGStab as Krylov.jl runs it (left preconditioner, shadow vector = b)."""


@dataclass(frozen=True)
class BornSeries:
    """The plain convergent Born series (Richardson iteration on the preconditioned system)."""


_ORTHO = {"mgs": L.FM_ORTHO_MGS, "cgs": L.FM_ORTHO_CGS, "cgs2": L.FM_ORTHO_CGS2, "block": L.FM_ORTHO_BLOCK}


def _device_available() -> int:
    return L.lib().fm_device_count()


class ConvergentBornSolver:
    """ConvergentBornSolver(resolution, grid_size, boundary_conditions, iterations_max=-1,
    tolerance=1e-6, linear_solver=KrylovJL_GMRES(), preconditioner="none", device="fmcuda")
    (convergent_born.jl:87-233).

    ``precision`` ("float64" / "float32" / "float32-math64": FP32 fields in HBM with FP64 arithmetic in the
    FFT, Green and potential kernels) replaces Julia's element-type parameter T; by default it is
    float32 when ``resolution`` holds numpy float32 values and float64 otherwise (the reference promotes
    the type of resolution and tolerance).  ``max_rhs`` bounds the batch held on the device at once.
    ``autotune=True`` picks launch shapes and the batch schedule for each batch shape on first use
    (fmcuda.autotune; cached on disk)."""

    def __init__(self, resolution: Sequence[float], grid_size: Sequence[int], boundary_conditions,
                 iterations_max: int = -1, tolerance: float = 1e-6, linear_solver=None,
                 preconditioner: str = "none", device: str = "fmcuda", precision: Optional[str] = None,
                 max_rhs: int = 64, device_index: int = 0, autotune: bool = False):
        if precision is None:
            precision = "float32" if all(isinstance(r, np.float32) for r in resolution) else "float64"
        if precision not in ("float32", "float64", "float32-math64"):
            raise ValueError("precision must be 'float32', 'float64' or 'float32-math64'")
        if device not in ("fmcuda", "cuda"):
            raise ValueError(f"GPU backend :{device} is not available. This package runs on the fmcuda "
                             f"(CUDA, sm_100a) backend only; it has no CPU path.")
        self.resolution = tuple(float(r) for r in resolution)
        self.grid_size = tuple(int(n) for n in grid_size)
        if isinstance(boundary_conditions, AbstractBoundaryCondition):
            boundary_conditions = (boundary_conditions,) * 3
        self.boundary_conditions = tuple(boundary_conditions)
        if len(self.boundary_conditions) != 3:
            raise ValueError("boundary_conditions must be one condition or three")
        if not all(r > 0 for r in self.resolution):
            raise ValueError("all resolution components must be positive")
        if not all(n > 0 for n in self.grid_size):
            raise ValueError("all grid_size components must be positive")
        if not (0 <= tolerance <= 1):
            raise ValueError("tolerance must be in [0, 1]")
        self.iterations_max = int(iterations_max)
        self.tolerance = float(tolerance)
        self.linear_solver = linear_solver if linear_solver is not None else KrylovJL_GMRES()
        self.preconditioner = preconditioner
        self.device = device
        self.precision = precision
        self.max_rhs = int(max_rhs)
        self.device_index = int(device_index)
        self.autotune = bool(autotune)
        self.backend = "fmcuda"
        self.Green_function = None
        self.Bornmax = 0
        self.iteration_count = 0
        self.residual_history: List[float] = []
        self.solver_state = None
        self.last_info: List[dict] = []
        self._plan: Optional[DevicePlan] = None

    # ---- configuration helpers (convergent_born.jl:250-260, 1012-1021) ----
    def padding(self):
        return tuple(padding_pixels(self.boundary_conditions[d], self.resolution[d]) for d in range(3))

    def padded_size(self):
        p = self.padding()
        return tuple(self.grid_size[d] + 2 * p[d] for d in range(3))

    def compute_ROI(self):
        p, g = self.padding(), self.grid_size
        return (p[0] + 1, p[0] + g[0], p[1] + 1, p[1] + g[1], p[2] + 1, p[2] + g[2])

    def plan(self) -> "DevicePlan":
        if self._plan is None:
            self._plan = DevicePlan(self.grid_size, self.padding(), self.resolution,
                                    [requires_averaging(bc) for bc in self.boundary_conditions],
                                    self.precision, self.max_rhs, self.device_index)
        return self._plan

    def release(self):
        if self._plan is not None:
            self._plan.destroy()
            self._plan = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def __repr__(self):
        return (f"ConvergentBornSolver{{{self.precision}}}: resolution={self.resolution} "
                f"grid_size={self.grid_size} iterations={self.iteration_count}")

    def solve_options(self, bornmax: int) -> L.fm_solve_opts:
        o = L.fm_solve_opts()
        ls = self.linear_solver
        if isinstance(ls, KrylovJL_GMRES):
            o.method = L.FM_METHOD_GMRES
            ortho = ls.ortho or ("mgs" if self.precision == "float64" else "cgs")
            o.ortho = _ORTHO[ortho]
            o.block = int(ls.block_size) if ortho == "block" else 0
            o.block_store = {"fp64": L.FM_BLOCK_FP64, "storage": L.FM_BLOCK_STORAGE,
                             "fp64-ortho": L.FM_BLOCK_FP64_ORTHO}[ls.block_vectors]
            o.restart = int(ls.gmres_restart)
        elif isinstance(ls, KrylovJL_BICGSTAB):
            o.method = L.FM_METHOD_BICGSTAB
        elif isinstance(ls, BornSeries):
            o.method = L.FM_METHOD_RICHARDSON
        else:
            raise ValueError(f"unsupported linear_solver {ls!r}")
        o.maxiters = max(bornmax * 2, 100)               # convergent_born.jl:746
        o.reltol = self.tolerance                         # :744
        o.abstol = self.tolerance * 1e-2                  # :745
        o.timeout_s = 0.0
        return o

    def attenuation_filters(self):
        return [np.ascontiguousarray(attenuation_filter(self.boundary_conditions[d], self.resolution[d],
                                                        self.grid_size[d])) for d in range(3)]


def reset(solver: ConvergentBornSolver) -> None:
    """reset! (convergent_born.jl:967-972)."""
    solver.iteration_count = 0
    solver.residual_history.clear()
    solver.solver_state = None


def compute_ROI(solver: ConvergentBornSolver):
    return solver.compute_ROI()


def grid_spacing(solver: ConvergentBornSolver):
    return solver.resolution


def domain_size(solver: ConvergentBornSolver):
    return tuple(solver.grid_size[i] * solver.resolution[i] for i in range(3))


class DevicePlan:
    """Owner of one fm_plan (device memory, stream, tables).  Also exposes the reference's
    internal seams (conv!, the CBS operator, the preconditioner, the curl) on host arrays."""

    def __init__(self, grid, pad, resolution, absorbing, precision: str, max_rhs: int, device: int = 0):
        lib = L.lib()
        if lib.fm_device_count() < 1:
            raise L.FMError(L.FM_ERR_CUDA, "no CUDA device is visible; fmcuda has no CPU path")
        d = L.fm_plan_desc()
        for a in range(3):
            d.grid[a] = int(grid[a])
            d.pad[a] = int(pad[a])
            d.resolution[a] = float(resolution[a])
            d.absorbing[a] = int(bool(absorbing[a]))
        d.precision = {"float64": L.FM_PREC_F64, "float32": L.FM_PREC_F32,
                       "float32-math64": L.FM_PREC_F32_MATH64}[precision]
        d.max_rhs = int(max_rhs)
        d.device = int(device)
        self.desc = d
        self.grid = tuple(int(g) for g in grid)
        self.pad = tuple(int(p) for p in pad)
        self.padded = tuple(self.grid[a] + 2 * self.pad[a] for a in range(3))
        self.handle = C.c_void_p()
        L.check(lib.fm_plan_create(C.byref(d), C.byref(self.handle)))

    def destroy(self):
        if self.handle:
            L.lib().fm_plan_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # -- helpers --
    def _field(self, a, nrhs=None) -> np.ndarray:
        a = np.asarray(a, dtype=np.complex128)
        shp = self.padded + (3,)
        if a.shape[:4] != shp:
            raise ValueError(f"field shape {a.shape} does not match padded grid {shp}")
        return np.asfortranarray(a)

    @staticmethod
    def _nrhs(a) -> int:
        return 1 if a.ndim == 4 else a.shape[4]

    # -- seams --
    def set_potential(self, V: np.ndarray, k_bg: float, eps_imag: float, wavelength: float):
        V = np.asfortranarray(np.asarray(V, dtype=np.complex128))
        if V.shape != self.padded:
            raise ValueError("potential must have the padded grid shape")
        L.check(L.lib().fm_set_potential(self.handle, L.ptr(V), k_bg, eps_imag, wavelength))

    def build_potential(self, eps: Optional[np.ndarray], eps_bg: float, wavelength: float, filters,
                        iterations_max: int):
        """_initialize_solver! on the device; eps None takes the permittivity fill_phantom painted there."""
        if eps is not None:
            eps = np.asfortranarray(np.asarray(eps, dtype=np.complex128))
            if eps.shape != self.grid:
                raise ValueError(f"medium grid_size {eps.shape} must match solver grid_size {self.grid}")
        info = L.fm_potential_info()
        fx, fy, fz = (np.ascontiguousarray(f, dtype=np.float64) for f in filters)
        L.check(L.lib().fm_build_potential(self.handle, None if eps is None else L.ptr(eps), eps_bg, wavelength,
                                           L.ptr(fx), L.ptr(fy), L.ptr(fz), int(iterations_max), C.byref(info)))
        return info

    def fill_phantom(self, shapes, eps_bg: float, copy_out: bool = False) -> Optional[np.ndarray]:
        """Paint ``shapes`` (medium.Shape, in order) over eps_bg into the plan's device permittivity."""
        arr = (L.fm_shape * max(1, len(shapes)))()
        for i, sh in enumerate(shapes):
            arr[i].kind = int(sh.kind)
            arr[i].axis = int(sh.axis)
            for a in range(3):
                arr[i].center[a] = float(sh.center[a])
            arr[i].radius = float(sh.radius)
            arr[i].extent = float(sh.extent)
            arr[i].value[0] = complex(sh.value).real
            arr[i].value[1] = complex(sh.value).imag
        out = np.empty(self.grid, dtype=np.complex128, order="F") if copy_out else None
        L.check(L.lib().fm_phantom_fill(self.handle, float(eps_bg), len(shapes), arr,
                                        None if out is None else L.ptr(out)))
        return out

    def green_apply(self, x: np.ndarray) -> np.ndarray:
        x = self._field(x)
        y = np.empty_like(x, order="F")
        L.check(L.lib().fm_green_apply(self.handle, self._nrhs(x), L.ptr(x), L.ptr(y)))
        return y

    def apply_operator(self, x: np.ndarray, y: Optional[np.ndarray] = None, alpha=1.0, beta=0.0) -> np.ndarray:
        x = self._field(x)
        y = np.zeros_like(x, order="F") if y is None else self._field(y).copy(order="F")
        a, b = complex(alpha), complex(beta)
        L.check(L.lib().fm_apply_operator(self.handle, self._nrhs(x), L.ptr(x), L.ptr(y), a.real, a.imag,
                                          b.real, b.imag))
        return y

    def apply_preconditioner(self, x: np.ndarray) -> np.ndarray:
        x = self._field(x)
        y = np.empty_like(x, order="F")
        L.check(L.lib().fm_apply_preconditioner(self.handle, self._nrhs(x), L.ptr(x), L.ptr(y)))
        return y

    def curl_field(self, E: np.ndarray) -> np.ndarray:
        E = self._field(E)
        H = np.empty_like(E, order="F")
        L.check(L.lib().fm_curl_field(self.handle, self._nrhs(E), L.ptr(E), L.ptr(H)))
        return H

    def solve_source(self, S: np.ndarray, opts: L.fm_solve_opts):
        S = self._field(S)
        n = self._nrhs(S)
        E = np.empty_like(S, order="F")
        H = np.empty_like(S, order="F")
        info = (L.fm_solve_info * n)()
        st = L.lib().fm_solve_source(self.handle, n, L.ptr(S), C.byref(opts), L.ptr(E), L.ptr(H), info)
        L.check(st, allow_not_converged=True)
        return E, H, list(info), st

    def solve_plane_waves(self, rhs_sources: List[List[PlaneWaveSource]], eps_bg: float, opts: L.fm_solve_opts,
                          keep_on_device: bool = False):
        n = len(rhs_sources)
        first = (C.c_int * (n + 1))()
        flat = []
        for b, srcs in enumerate(rhs_sources):
            first[b] = len(flat)
            flat.extend(srcs)
        first[n] = len(flat)
        arr = (L.fm_plane_wave * len(flat))()
        for i, s in enumerate(flat):
            arr[i].wavelength = s.wavelength
            for a in range(3):
                arr[i].polarization[2 * a] = s.polarization[a].real
                arr[i].polarization[2 * a + 1] = s.polarization[a].imag
                arr[i].k_vector[a] = s.k_vector[a]
            arr[i].amplitude = s.amplitude
            arr[i].phase = s.phase
        info = (L.fm_solve_info * n)()
        if keep_on_device:
            st = L.lib().fm_solve_plane_waves(self.handle, n, first, arr, eps_bg, C.byref(opts), None, None, info)
            L.check(st, allow_not_converged=True)
            return None, None, list(info), st
        shp = self.grid + (3, n)
        E = np.empty(shp, dtype=np.complex128, order="F")
        H = np.empty(shp, dtype=np.complex128, order="F")
        st = L.lib().fm_solve_plane_waves(self.handle, n, first, arr, eps_bg, C.byref(opts), L.ptr(E), L.ptr(H),
                                          info)
        L.check(st, allow_not_converged=True)
        return E, H, list(info), st

    # -- instrumentation --
    def set_profiling(self, on: bool):
        L.check(L.lib().fm_set_profiling(self.handle, int(bool(on))))

    def kernel_stats(self):
        arr = (L.fm_kernel_stat * 16)()
        n = L.lib().fm_kernel_stats(self.handle, arr, 16)
        return {arr[i].name.decode(): dict(launches=arr[i].launches, ms=arr[i].ms, bytes=arr[i].bytes)
                for i in range(max(n, 0))}

    def launch_count(self) -> int:
        return int(L.lib().fm_launch_count(self.handle))

    def stream(self) -> int:
        return int(L.lib().fm_stream(self.handle) or 0)

    def synchronize(self):
        L.check(L.lib().fm_synchronize(self.handle))

    def copy_fields(self, n: int):
        shp = self.grid + (3, n)
        E = np.empty(shp, dtype=np.complex128, order="F")
        H = np.empty(shp, dtype=np.complex128, order="F")
        L.check(L.lib().fm_copy_fields(self.handle, n, L.ptr(E), L.ptr(H)))
        return E, H


def _prepare(solver: ConvergentBornSolver, medium: Medium, wavelength: float):
    if medium_grid_size(medium) != solver.grid_size:
        raise ValueError(f"medium grid_size {medium_grid_size(medium)} must match solver grid_size "
                         f"{solver.grid_size}")
    plan = solver.plan()
    eps = None
    if isinstance(medium, DevicePhantom):  # painted on the device: no permittivity crosses from the host
        plan.fill_phantom(medium.shapes, medium.permittivity_bg)
    else:
        eps = medium.permittivity
    info = plan.build_potential(eps, medium.permittivity_bg, wavelength, solver.attenuation_filters(),
                                solver.iterations_max)
    solver.Bornmax = int(info.bornmax)
    solver.iteration_count = 0
    solver.residual_history.clear()
    if solver.Bornmax < 1:
        raise ValueError("Bornmax < 1: iterations_max must be negative (auto) or >= 1")
    return plan, info


def _record(solver: ConvergentBornSolver, infos, status: int):
    solver.last_info = [dict(iterations=i.iterations, solved=bool(i.solved), residual=i.residual,
                             residual0=i.residual0) for i in infos]
    solver.iteration_count = int(infos[-1].iterations)
    solver.residual_history.append(float(infos[-1].residual))
    if status == L.FM_NOT_CONVERGED:
        L.warn_not_converged()


def solve(solver: ConvergentBornSolver, sources, medium: Medium) -> ElectromagneticField:
    """LinearSolve.solve(solver, sources, medium) (convergent_born.jl:565-600), on the GPU."""
    wl = source_wavelength(sources)
    srcs = as_list(sources)
    plan, _ = _prepare(solver, medium, wl)
    E, H, infos, st = plan.solve_plane_waves([srcs], medium.permittivity_bg, solver.solve_options(solver.Bornmax))
    _record(solver, infos, st)
    return ElectromagneticField(np.asfortranarray(E[..., 0]), np.asfortranarray(H[..., 0]), solver.resolution, wl)


def solve_batch(solver: ConvergentBornSolver, sources_list: Sequence, medium: Medium) -> List[ElectromagneticField]:
    """Independent solves of one medium for many illuminations, as one batched GPU solve (new).

    Entry b of ``sources_list`` is what ``solve`` would take (one source or a coherent list); the
    result b equals ``solve(solver, sources_list[b], medium)``."""
    lists = [as_list(s) for s in sources_list]
    if not lists:
        raise ValueError("sources_list cannot be empty")
    wl = source_wavelength(lists[0])
    for s in lists:
        if source_wavelength(s) != wl:
            raise ValueError("all right-hand sides must share the wavelength of the potential")
    if solver.autotune:
        from . import autotune as AT
        AT.configure(solver, AT.autotune(solver, lists, medium))
    plan, _ = _prepare(solver, medium, wl)
    E, H, infos, st = plan.solve_plane_waves(lists, medium.permittivity_bg, solver.solve_options(solver.Bornmax))
    _record(solver, infos, st)
    return [ElectromagneticField(np.asfortranarray(E[..., b]), np.asfortranarray(H[..., b]), solver.resolution, wl)
            for b in range(len(lists))]
