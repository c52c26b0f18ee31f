"""Continuous-batching request loop on the slot engine (fm_engine_* in include/fmcuda.h).

New: the reference solves one request per ``solve`` call.  Here requests (a permittivity, 1..n plane-wave
illuminations, a tolerance) of mixed grid shapes are served concurrently:

* one engine per grid shape, its slot count sized from a device-memory budget split across the shapes;
* a request's right-hand sides queue on their shape's engine and are admitted into slots as slots free
  up; every engine step advances all running right-hand sides by one GMRES iteration in shared launches
  (continuous batching at iteration granularity), or, with ``ortho="block"``, by one s-step block of 8
  iterations (block GMRES on FP64 block vectors, as the batched solve runs it; restarted when the basis is
  full);
* each shape's engine is stepped by its own host thread on its own CUDA stream, so shapes overlap on the
  device;
* per-request latency (arrival to completion of its last right-hand side) and throughput are recorded.

Each right-hand side runs the iteration of ``solve`` (GMRES with warm start b and the same stopping test,
restarted every ``basis`` iterations when its iteration limit exceeds the basis), so a request's result
does not depend on what else is in flight.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L
from .boundary import AbsorbingBoundaryCondition, PeriodicBoundaryCondition, TanhProfile
from .fields import ElectromagneticField
from .medium import Medium, phantom_random_beads
from .solver import ConvergentBornSolver, DevicePlan
from .sources import PlaneWaveSource, illumination_cone

_ORTHO = {"cgs": L.FM_ORTHO_CGS, "cgs2": L.FM_ORTHO_CGS2, "block": L.FM_ORTHO_BLOCK}


@dataclass
class Request:
    req_id: int
    medium: Medium
    sources: List[PlaneWaveSource]
    tolerance: float = 1e-5
    arrival: float = 0.0       # offset from the start of a run, seconds
    submitted: float = 0.0     # perf_counter at submission
    finished: float = 0.0      # perf_counter when the last right-hand side completed
    E: Optional[np.ndarray] = None
    H: Optional[np.ndarray] = None
    infos: Dict[int, dict] = field(default_factory=dict)
    done_event: threading.Event = field(default_factory=threading.Event)

    @property
    def shape(self) -> Tuple[int, int, int]:
        return tuple(self.medium.permittivity.shape)

    @property
    def latency(self) -> float:
        return self.finished - self.submitted

    def field(self, rhs: int, resolution) -> ElectromagneticField:
        return ElectromagneticField(np.asfortranarray(self.E[..., rhs]), np.asfortranarray(self.H[..., rhs]),
                                    resolution, self.sources[rhs].wavelength)


def engine_slot_bytes(solver: ConvergentBornSolver, basis: int, ortho: str = "cgs") -> int:
    """Device bytes one slot of an engine on ``solver``'s grid holds (fm_engine_slot_bytes_ortho)."""
    return int(L.lib().fm_engine_slot_bytes_ortho(C.byref(solver.plan().desc), int(basis), _ORTHO[ortho]))


class Engine:
    """One fm_engine (``slots`` right-hand sides in flight) on the plan of ``solver``."""

    def __init__(self, solver: ConvergentBornSolver, slots: int, basis: int = 100, wavelength: float = 500e-9,
                 permittivity_bg: float = 1.33 ** 2, ortho: str = "cgs"):
        self.solver = solver
        self.plan: DevicePlan = solver.plan()
        self._filters = solver.attenuation_filters()
        f = self._filters
        self.handle = C.c_void_p()
        L.check(L.lib().fm_engine_create(self.plan.handle, int(slots), int(basis), float(wavelength),
                                         float(permittivity_bg), L.ptr(f[0]), L.ptr(f[1]), L.ptr(f[2]),
                                         _ORTHO[ortho], C.byref(self.handle)))
        self.slots = int(slots)
        self.basis = int(basis)
        self.grid = solver.grid_size
        self._keep: Dict[int, tuple] = {}
        self._lock = threading.Lock()

    def submit(self, req: Request, iterations_max: Optional[int] = None):
        """Queue every right-hand side of ``req``; results land in req.E / req.H (grid x 3 x nrhs).
        ``iterations_max`` overrides the solver's setting (Bornmax when >= 0) for this request."""
        g = self.grid
        eps = np.asfortranarray(req.medium.permittivity, dtype=np.complex128)
        n = len(req.sources)
        req.E = np.empty(g + (3, n), dtype=np.complex128, order="F")
        req.H = np.empty(g + (3, n), dtype=np.complex128, order="F")
        arr = (L.fm_plane_wave * n)()
        for i, s in enumerate(req.sources):
            arr[i].wavelength = s.wavelength
            for a in range(3):
                arr[i].polarization[2 * a] = s.polarization[a].real
                arr[i].polarization[2 * a + 1] = s.polarization[a].imag
                arr[i].k_vector[a] = s.k_vector[a]
            arr[i].amplitude = s.amplitude
            arr[i].phase = s.phase
        with self._lock:
            self._keep[req.req_id] = (req, eps, arr)
        req.submitted = time.perf_counter()
        itmax = self.solver.iterations_max if iterations_max is None else int(iterations_max)
        st = L.lib().fm_engine_submit(self.handle, req.req_id, L.ptr(eps), n, arr, req.tolerance, itmax,
                                      L.ptr(req.E), L.ptr(req.H))
        if st != L.FM_OK:
            with self._lock:
                del self._keep[req.req_id]
            L.check(st)

    def step(self) -> List[Tuple[int, int, dict]]:
        nd = C.c_int(0)
        reqs = (C.c_longlong * self.slots)()
        rhs = (C.c_int * self.slots)()
        info = (L.fm_solve_info * self.slots)()
        L.check(L.lib().fm_engine_step(self.handle, C.byref(nd), reqs, rhs, info, self.slots))
        return [(int(reqs[k]), int(rhs[k]), dict(iterations=int(info[k].iterations), solved=bool(info[k].solved),
                                                  residual=float(info[k].residual),
                                                  residual0=float(info[k].residual0)))
                for k in range(nd.value)]

    def status(self) -> Tuple[int, int]:
        r, q = C.c_int(0), C.c_int(0)
        L.check(L.lib().fm_engine_status(self.handle, C.byref(r), C.byref(q)))
        return r.value, q.value

    def complete(self, req_id: int, rhs: int, info: dict) -> Optional[Request]:
        """Record one finished right-hand side; returns the request once all of its right-hand sides are in."""
        with self._lock:
            req = self._keep[req_id][0]
            req.infos[rhs] = info
            if len(req.infos) == len(req.sources):
                req.finished = time.perf_counter()
                del self._keep[req_id]
                return req
        return None

    def drain(self, reqs: Sequence[Request], max_steps: int = 100000):
        """Step until every request in ``reqs`` is complete (single-threaded use)."""
        left = {r.req_id for r in reqs}
        for _ in range(max_steps):
            if not left:
                return
            for req_id, rhs, info in self.step():
                r = self.complete(req_id, rhs, info)
                if r is not None:
                    r.done_event.set()
                    left.discard(r.req_id)
        raise RuntimeError("engine did not finish within max_steps")

    def close(self):
        if self.handle:
            L.lib().fm_engine_destroy(self.handle)
            self.handle = C.c_void_p()


def serving_boundaries(shape) -> tuple:
    """Periodic x, y; absorbing z with thickness = attenuation thickness = Nz * 50 nm (padded z = 2 Nz)."""
    t = shape[2] * 50e-9
    return (PeriodicBoundaryCondition(), PeriodicBoundaryCondition(),
            AbsorbingBoundaryCondition(thickness=t, attenuation_thickness=t, sharpness=1.0, profile=TanhProfile))


def slot_plan(shapes: Sequence[Tuple[int, int, int]], budget_bytes: float, basis: int, precision: str,
              resolution=(50e-9,) * 3, max_slots: int = 64, target_elements: float = 48e6, ortho: str = "cgs"
              ) -> Dict[Tuple[int, int, int], int]:
    """Slots per shape under one device-memory budget.

    The Born-iteration kernels are bandwidth-bound and fill the GPU once one launch streams about
    ``target_elements`` complex values (one padded 256^3 three-component field), so each shape asks for
    the slots that make one field batch that large (small grids batch many right-hand sides, a 256^3
    grid one).  Every shape gets one slot; when the remaining asks exceed the rest of the budget they are
    scaled down in proportion."""
    per, want = {}, {}
    for s in shapes:
        sv = ConvergentBornSolver(resolution=resolution, grid_size=s, boundary_conditions=serving_boundaries(s),
                                  precision=precision, max_rhs=1)
        d = L.fm_plan_desc()
        d.grid[:] = list(s)
        d.pad[:] = list(sv.padding())
        d.precision = {"float64": L.FM_PREC_F64, "float32": L.FM_PREC_F32,
                       "float32-math64": L.FM_PREC_F32_MATH64}[precision]
        per[tuple(s)] = int(L.lib().fm_engine_slot_bytes_ortho(C.byref(d), int(basis), _ORTHO[ortho]))
        field = 3.0 * float(np.prod(sv.padded_size()))
        want[tuple(s)] = int(min(max_slots, max(1, np.ceil(target_elements / field))))
    base = sum(per.values())                     # one slot per shape first
    extra = sum((want[s] - 1) * per[s] for s in want)
    f = 0.0 if extra == 0 or budget_bytes <= base else min(1.0, (budget_bytes - base) / extra)
    return {s: 1 + int(np.floor((want[s] - 1) * f)) for s in want}


class Server:
    """Serves requests of several grid shapes with one engine (and one stepping thread) per shape."""

    def __init__(self, shapes: Sequence[Tuple[int, int, int]], budget_bytes: float = 150e9,
                 precision: str = "float32-math64", basis: int = 100, wavelength: float = 500e-9,
                 permittivity_bg: float = 1.33 ** 2, resolution=(50e-9,) * 3, max_slots: int = 64,
                 slots: Optional[Dict[Tuple[int, int, int], int]] = None, ortho: str = "cgs"):
        self.resolution = tuple(resolution)
        self.slots = dict(slots) if slots is not None else slot_plan(shapes, budget_bytes, basis, precision,
                                                                     resolution, max_slots, ortho=ortho)
        self.engines: Dict[Tuple[int, int, int], Engine] = {}
        for shape in shapes:
            shape = tuple(shape)
            solver = ConvergentBornSolver(resolution=resolution, grid_size=shape,
                                          boundary_conditions=serving_boundaries(shape), precision=precision,
                                          max_rhs=self.slots[shape])
            self.engines[shape] = Engine(solver, self.slots[shape], basis, wavelength, permittivity_bg, ortho)
        self._threads: List[threading.Thread] = []
        self._stop = threading.Event()
        self._work = {k: threading.Event() for k in self.engines}
        self.completed: List[Request] = []
        self._clock = threading.Lock()
        self.errors: List[BaseException] = []
        self.steps = {k: 0 for k in self.engines}

    def start(self):
        for shape, eng in self.engines.items():
            t = threading.Thread(target=self._run, args=(shape, eng), daemon=True)
            t.start()
            self._threads.append(t)

    def _run(self, shape, eng: Engine):
        try:
            while not self._stop.is_set():
                running, queued = eng.status()
                if running == 0 and queued == 0:
                    self._work[shape].wait(0.001)
                    self._work[shape].clear()
                    continue
                done = eng.step()
                self.steps[shape] += 1
                for req_id, rhs, info in done:
                    req = eng.complete(req_id, rhs, info)
                    if req is not None:
                        with self._clock:
                            self.completed.append(req)
                        req.done_event.set()
        except BaseException as e:  # surfaced by wait()
            self.errors.append(e)
            self._stop.set()

    def submit(self, req: Request):
        self.engines[req.shape].submit(req)
        self._work[req.shape].set()

    def wait(self, reqs: Sequence[Request], timeout: float = 3600.0):
        t0 = time.perf_counter()
        for r in reqs:
            while not r.done_event.wait(0.05):
                if self.errors:
                    raise self.errors[0]
                if time.perf_counter() - t0 > timeout:
                    raise TimeoutError(f"request {r.req_id} not finished")
        if self.errors:
            raise self.errors[0]

    def stop(self):
        self._stop.set()
        for t in self._threads:
            t.join(timeout=60)
        for e in self.engines.values():
            e.close()
        for e in self.engines.values():
            e.solver.release()

    def __enter__(self):
        self.start()
        return self

    def __exit__(self, *a):
        self.stop()


SERVING_SHAPES = ((64, 64, 32), (96, 96, 64), (128, 128, 64), (256, 256, 128))


def serving_requests(n: int, rate: float = 200.0, shapes=SERVING_SHAPES, max_angles: int = 32, seed: int = 7,
                     wavelength: float = 500e-9, permittivity_bg: float = 1.33 ** 2, resolution=(50e-9,) * 3,
                     tolerance: float = 1e-5, na: float = 1.2, beads: int = 12, radius_range=(4, 12),
                     index_range=(1.36, 1.60)) -> List[Request]:
    """A seeded Poisson request stream: exponential inter-arrival times of mean 1/rate, grid drawn
    uniformly from ``shapes``, 1..max_angles illumination angles (uniform; polarisation s and p
    alternating), phantom of ``beads`` non-overlapping beads (radius U[radius_range] px, index
    U[index_range]) in the background medium."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        shape = tuple(shapes[int(rng.integers(len(shapes)))])
        na_ = int(rng.integers(1, max_angles + 1))
        pseed = int(rng.integers(1 << 30))
        med = phantom_random_beads(shape, beads, radius_range, index_range, permittivity_bg, pseed)
        cone = illumination_cone(shape, resolution, wavelength, permittivity_bg, na_, na, pseed)
        srcs = [cone[2 * a + (a & 1)] for a in range(na_)]
        out.append(Request(req_id=i, medium=med, sources=srcs, tolerance=tolerance, arrival=t))
    return out


def run_stream(server: Server, requests: Sequence[Request], timeout: float = 3600.0) -> dict:
    """Submit ``requests`` at their arrival offsets, wait for all, and summarise latency and throughput."""
    t0 = time.perf_counter()
    for r in requests:
        dt = r.arrival - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        server.submit(r)
    server.wait(requests, timeout)
    t1 = max(r.finished for r in requests)
    lat = np.array([r.latency for r in requests])
    nrhs = sum(len(r.sources) for r in requests)
    iters = sum(i["iterations"] for r in requests for i in r.infos.values())
    # Born iterations weighted by the padded voxel count of their grid: comparable across grid shapes and with
    # the batched solve (born_iterations_per_s x padded voxels there)
    padded = {k: float(np.prod(e.solver.padded_size())) for k, e in server.engines.items()}
    vox_iters = sum(i["iterations"] * padded[tuple(np.shape(r.medium.permittivity))]
                    for r in requests for i in r.infos.values())
    return {"requests": len(requests), "solves": nrhs, "wall_s": t1 - t0, "solves_per_s": nrhs / (t1 - t0),
            "requests_per_s": len(requests) / (t1 - t0), "born_iterations_per_s": iters / (t1 - t0),
            "padded_voxel_iterations_per_s": vox_iters / (t1 - t0),
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "offered_rate": len(requests) / max(requests[-1].arrival, 1e-9),
            "converged": sum(i["solved"] for r in requests for i in r.infos.values()),
            "slots": {"x".join(map(str, k)): v for k, v in server.slots.items()}}
