"""Autotuner on the GPU: every launch knob leaves the result unchanged, invalid values are rejected, and an
autotuned batch solve matches the untuned one."""
import ctypes
import warnings

import numpy as np
import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, bead, configs, random_field, rel
from oracle import cbs_oracle as O

import fmcuda as F
from fmcuda import _lib
from fmcuda import autotune as AT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_launch_knobs_do_not_change_the_operator(precision):
    grid = (32, 32, 16)
    ocfg, solver = configs(grid, absorbing_z(grid[2]), precision=precision)
    pot = O.build_potential(ocfg, bead(grid, 4.0), EPS_BG, WL)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    x = random_field(ocfg.padded_size + (3, 3), 21)
    ref = plan.apply_operator(x)
    tol = 1e-13 if precision == "float64" else 1e-7
    for cfg in ({"tma_y": 0}, {"tma_z": 0}, {"tma_ctas": 1}, {"row_threads": 128}, {"tma_y": 0, "tma_z": 0},
                {"tma_ctas": 2, "row_threads": 128}):
        AT.apply(plan, dict(AT.DEFAULT, **cfg))
        assert AT.read(plan) == {k: v for k, v in dict(AT.DEFAULT, **cfg).items() if k != "block"}
        assert rel(plan.apply_operator(x), ref) < tol
    AT.apply(plan, AT.DEFAULT)
    solver.release()


def test_invalid_tuning_values_rejected():
    grid = (16, 16, 8)
    ocfg, solver = configs(grid, absorbing_z(8))
    plan = solver.plan()
    lib = _lib.lib()
    for knob, value in ((_lib.FM_TUNE_Y_TMA, 2), (_lib.FM_TUNE_ROW_THREADS, 512), (_lib.FM_TUNE_TMA_CTAS_PER_SM, -1),
                        (_lib.FM_TUNE_WAVE_RHS, -3), (_lib.FM_TUNE_BLOCK_DOT, 3), (99, 0)):
        assert lib.fm_plan_set_tuning(plan.handle, knob, value) == _lib.FM_ERR_INVALID
    v = ctypes.c_int(-1)
    assert lib.fm_plan_get_tuning(plan.handle, _lib.FM_TUNE_ROW_THREADS, ctypes.byref(v)) == _lib.FM_OK
    assert v.value == 256
    solver.release()


def test_autotuned_solve_batch_matches_untuned(tmp_path, monkeypatch):
    monkeypatch.setenv("FMCUDA_CACHE", str(tmp_path / "tune.json"))
    grid = (32, 32, 16)
    srcs = F.illumination_cone(grid, RES, WL, EPS_BG, 3, 1.2, 5)
    med = F.Medium(bead(grid, 4.0), EPS_BG)
    outs = {}
    for tuned in (False, True):
        solver = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=absorbing_z(16)[1],
                                        precision="float32-math64", autotune=tuned, max_rhs=8,
                                        linear_solver=F.KrylovJL_GMRES(ortho="block", block_size=8))
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            outs[tuned] = F.solve_batch(solver, [[s] for s in srcs], med)
        if tuned:
            key = AT.cache_key(solver, len(srcs), "block")
            cfg = AT._load()[key]
            assert cfg["trials"] >= 2 and cfg["block"] in (4, 8)
            assert AT.read(solver.plan())["row_threads"] == cfg["row_threads"]
        solver.release()
    for a, b in zip(outs[True], outs[False]):
        assert rel(a.E, b.E) < 1e-5
        assert rel(a.H, b.H) < 1e-5


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_waves_and_host_output_copies(precision):
    """Right-hand sides solved in waves of one (three waves, the two device output slots used in turn while the
    copy of the previous wave to the host overlaps the next wave) equal the same batch in one wave."""
    grid = (16, 16, 8)
    ocfg, solver = configs(grid, absorbing_z(8), precision=precision,
                           linear_solver=F.KrylovJL_GMRES(ortho="block", block_size=4))
    med = F.Medium(bead(grid, 3.0), EPS_BG)
    srcs = F.illumination_cone(grid, RES, WL, EPS_BG, 2, 1.2, 3)[:3]
    outs = {}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        for w in (0, 1):
            AT.apply(solver.plan(), {"wave_rhs": w})
            outs[w] = F.solve_batch(solver, [[s] for s in srcs], med)
    AT.apply(solver.plan(), {"wave_rhs": 0})
    tol = 1e-12 if precision == "float64" else 1e-6
    for a, b in zip(outs[1], outs[0]):
        assert np.all(np.isfinite(a.E)) and np.all(np.isfinite(a.H))
        assert rel(a.E, b.E) < tol
        assert rel(a.H, b.H) < tol
    solver.release()
