"""Autotuner of launch shapes and batch schedules (new; not in the reference).

The knobs change how the solve is launched, never what it computes (up to rounding: the block size of block
GMRES changes the order of the Gram-Schmidt arithmetic, and every candidate keeps the accuracy bar):

* ``tma_y``, ``tma_z``   -- TMA-staged (tile) y / z FFT passes or the register-only ones (fm_plan_set_tuning)
* ``tma_ctas``           -- persistent CTAs per SM of the TMA passes (0 = occupancy limit)
* ``row_threads``        -- threads per block of the x and y row passes (128 or 256)
* ``wave_rhs``           -- right-hand sides per wave (0 = as many as device memory holds)
* ``block_dot``          -- block dot of block GMRES: bulk-copy pipeline (1) or register-staged kernel (0)
* ``block``              -- vectors per block of block GMRES (8 or 4)

``autotune`` times short fixed-work solves of the caller's own batch (tolerance 0, a few iterations) on the
device (best of 3), changes one knob at a time from the current best (coordinate search, two sweeps), and keeps
a change only when it is more than 2 % faster.  Results are cached per device, grid, padding, precision, batch size and Gram-Schmidt variant, in
memory and in a JSON file (``$FMCUDA_CACHE`` or ``~/.cache/fmcuda/autotune.json``).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
import time
import warnings
from typing import Callable, Dict, List, Optional, Sequence

from . import _lib as L

DEFAULT = {"tma_y": 1, "tma_z": 1, "tma_ctas": 0, "row_threads": 256, "wave_rhs": 0, "block_dot": 0, "block": 8}
# block_dot is not searched: the trials run a few iterations (a basis of a few vectors) and did not separate the
# two kernels, while over a full solve of 100 iterations the register-staged one is faster
SPACE = {"tma_y": (1, 0), "tma_z": (1, 0), "tma_ctas": (0, 1, 2), "row_threads": (256, 128), "block": (8, 4)}
_KNOB = {"tma_y": L.FM_TUNE_Y_TMA, "tma_z": L.FM_TUNE_Z_TMA, "tma_ctas": L.FM_TUNE_TMA_CTAS_PER_SM,
         "row_threads": L.FM_TUNE_ROW_THREADS, "wave_rhs": L.FM_TUNE_WAVE_RHS, "block_dot": L.FM_TUNE_BLOCK_DOT}
_memory: Dict[str, dict] = {}
_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("FMCUDA_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "fmcuda",
                                                          "autotune.json")


def device_name(index: int = 0) -> str:
    try:
        import pynvml
        pynvml.nvmlInit()
        name = pynvml.nvmlDeviceGetName(pynvml.nvmlDeviceGetHandleByIndex(index))
        return name.decode() if isinstance(name, bytes) else str(name)
    except Exception:
        return "cuda"


def cache_key(solver, nrhs: int, ortho: str, device: Optional[str] = None) -> str:
    return "|".join([device or device_name(solver.device_index), "x".join(map(str, solver.grid_size)),
                     "x".join(map(str, solver.padding())), solver.precision, str(int(nrhs)), ortho])


def _load() -> Dict[str, dict]:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(key: str, cfg: dict):
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        data = _load()
        data[key] = cfg
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home keeps the in-memory cache only


def apply(plan, cfg: dict):
    """Set the launch knobs of ``cfg`` on a DevicePlan."""
    for k, knob in _KNOB.items():
        if k in cfg:
            L.check(L.lib().fm_plan_set_tuning(plan.handle, knob, int(cfg[k])))


def read(plan) -> dict:
    out = {}
    for k, knob in _KNOB.items():
        v = C.c_int(0)
        L.check(L.lib().fm_plan_get_tuning(plan.handle, knob, C.byref(v)))
        out[k] = v.value
    return out


# a knob changes only for a gain above the trials' run-to-run spread (about 1 % for one-second trials)
MIN_GAIN = 0.02


def coordinate_search(measure: Callable[[dict], float], start: dict, space: Dict[str, Sequence],
                      sweeps: int = 2) -> (dict, Dict[str, float]):
    """Greedy search: from ``start``, try each alternative value of one knob at a time and keep any
    improvement; repeat ``sweeps`` times or until nothing improves.  ``measure`` returns seconds."""
    best = dict(start)
    seen: Dict[str, float] = {}

    def timed(cfg):
        key = json.dumps(cfg, sort_keys=True)
        if key not in seen:
            seen[key] = measure(cfg)
        return seen[key]

    t_best = timed(best)
    for _ in range(sweeps):
        improved = False
        for knob, values in space.items():
            for v in values:
                if v == best.get(knob):
                    continue
                cand = dict(best)
                cand[knob] = v
                t = timed(cand)
                if t < t_best * (1.0 - MIN_GAIN):
                    best, t_best, improved = cand, t, True
        if not improved:
            break
    return best, seen


def autotune(solver, sources_list, medium, trial_iters: Optional[int] = None, use_cache: bool = True,
             sweeps: int = 2) -> dict:
    """Pick the launch shapes and batch schedule for ``solve_batch(solver, sources_list, medium)``."""
    from .solver import KrylovJL_GMRES, _prepare
    from .sources import as_list, source_wavelength
    lists = [as_list(s) for s in sources_list]
    ls = solver.linear_solver
    ortho = (ls.ortho or ("mgs" if solver.precision == "float64" else "cgs")) if isinstance(ls, KrylovJL_GMRES) \
        else type(ls).__name__
    key = cache_key(solver, len(lists), ortho)
    with _lock:
        if use_cache:
            if key in _memory:
                return dict(_memory[key])
            disk = _load().get(key)
            if disk:
                _memory[key] = disk
                return dict(disk)
    wl = source_wavelength(lists[0])
    plan, info = _prepare(solver, medium, wl)
    opts = solver.solve_options(solver.Bornmax)
    space = {k: v for k, v in SPACE.items() if k != "block" or ortho == "block"}
    block0 = getattr(ls, "block_size", 4)
    it = trial_iters or (max(3, 2 * block0 + 2 * block0) if ortho == "block" else 12)
    opts.maxiters = it
    opts.reltol = 0.0
    opts.abstol = 0.0

    def measure(cfg):
        apply(plan, cfg)
        if ortho == "block":
            opts.block = int(cfg.get("block", block0))
        best = float("inf")
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            for _ in range(3):
                plan.synchronize()
                t0 = time.perf_counter()
                plan.solve_plane_waves(lists, medium.permittivity_bg, opts, keep_on_device=True)
                plan.synchronize()
                best = min(best, time.perf_counter() - t0)
        return best

    start = dict(DEFAULT)
    start["block"] = block0
    best, seen = coordinate_search(measure, start, space, sweeps)
    best = dict(best)
    best["seconds_per_trial"] = min(seen.values())
    best["trials"] = len(seen)
    apply(plan, best)
    with _lock:
        _memory[key] = best
    if use_cache:
        _store(key, best)
    return dict(best)


def configure(solver, cfg: dict):
    """Apply a tuned configuration to ``solver`` (its plan's launch knobs and its block size)."""
    apply(solver.plan(), cfg)
    ls = solver.linear_solver
    if "block" in cfg and getattr(ls, "ortho", None) == "block":
        from dataclasses import replace
        solver.linear_solver = replace(ls, block_size=int(cfg["block"]))
