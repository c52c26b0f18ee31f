"""General padded axis lengths (odd, non-powers of two): the reference accepts any grid, e.g. the 201 x 201 x 191
grid of examples/two_beam_interference.jl:50 (padded z 197 by its 300 nm absorbing boundary).  Such plans run
the general passes (Bluestein's algorithm per axis, plain Green / curl passes); the Green and curl k-index formulas
differ for odd N (src/core/dyadic_green.jl:203-208 vs src/core/curl.jl:84-86), and both are exercised here.

Tolerances: FP64 <= 1e-12 for single applications and <= 1e-10 for solves (with the oracle's iteration count);
FP32 storage with FP64 arithmetic 2e-7 / 1e-5; all-FP32 arithmetic 2e-6 / 1e-5.
"""
import warnings

import numpy as np
import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, bead, configs, periodic, random_field, rel, xpol
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu

OP_TOL = {"float64": 1e-12, "float32": 2e-6, "float32-math64": 2e-7}
SOLVE_TOL = {"float64": 1e-10, "float32": 1e-5, "float32-math64": 1e-5}


def absorbing_all(grid):
    ob, fb = [], []
    for d in range(3):
        t = grid[d] * RES[d]
        ob.append(O.AbsorbingBC(t, t, 1.0, O.TANH))
        fb.append(F.AbsorbingBoundaryCondition(thickness=t, attenuation_thickness=t, sharpness=1.0,
                                               profile=F.TanhProfile))
    return tuple(ob), tuple(fb)


def _bcs(kind, grid):
    return {"per": periodic, "absz": lambda: absorbing_z(grid[2]), "all": lambda: absorbing_all(grid)}[kind]()


CASES = [((15, 12, 10), "per"), ((9, 20, 7), "absz"), ((12, 10, 6), "all"), ((24, 17, 33), "absz"), ((5, 7, 3), "per")]


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
@pytest.mark.parametrize("grid,kind", CASES)
def test_green_operator_curl_general_sizes(precision, grid, kind):
    ocfg, solver = configs(grid, _bcs(kind, grid), precision=precision)
    eps = bead(grid, max(1.5, min(grid) / 4))
    pot = O.build_potential(ocfg, eps, EPS_BG, WL)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    x = random_field(ocfg.padded_size + (3,), 31)
    assert rel(plan.green_apply(x), O.green_conv(x, ocfg, pot.k_square)) < OP_TOL[precision]
    y0 = random_field(ocfg.padded_size + (3,), 32)
    ref = O.cbs_operator(x, pot.V, ocfg, pot.k_square, alpha=0.9 - 0.1j, beta=0.3 + 0.2j, y=y0)
    assert rel(plan.apply_operator(x, y0, alpha=0.9 - 0.1j, beta=0.3 + 0.2j), ref) < OP_TOL[precision]
    assert rel(plan.apply_preconditioner(x), O.cbs_preconditioner(x, pot.V, pot.eps_imag)) < OP_TOL[precision]
    assert rel(plan.curl_field(x), O.magnetic_field(x, RES, WL)) < OP_TOL[precision]
    solver.release()


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
@pytest.mark.parametrize("grid,kind", [((15, 13, 9), "absz"), ((12, 10, 6), "all")])
def test_solve_general_sizes(precision, grid, kind):
    ls = F.KrylovJL_GMRES(ortho="mgs" if precision == "float64" else "cgs")
    ocfg, solver = configs(grid, _bcs(kind, grid), precision=precision, linear_solver=ls)
    eps = bead(grid, 3.0)
    osrc, fsrc = xpol()
    ref = O.solve(ocfg, osrc, eps, EPS_BG)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, fsrc, F.Medium(eps, EPS_BG))
    assert out.E.shape == grid + (3,)
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
    assert rel(out.E, ref.E) < SOLVE_TOL[precision]
    assert rel(out.H, ref.H) < SOLVE_TOL[precision]
    solver.release()


def test_two_beam_example_grid_operator_fp64():
    """The reference example's grid: 201 x 201 x 191 at 50 nm, absorbing z of 300 nm (padded 201 x 201 x 197),
    water at n 1.333, 532 nm (examples/two_beam_interference.jl:40-60): one Green application and one operator
    application against the oracle."""
    grid = (201, 201, 191)
    t = 300e-9
    ob = (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(t, t, 1.0, O.TANH))
    fb = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(),
          F.AbsorbingBoundaryCondition(thickness=t, attenuation_thickness=t, sharpness=1.0, profile=F.TanhProfile))
    eps_bg = 1.333 ** 2
    wl = 532e-9
    ocfg = O.SolverConfig(RES, grid, ob)
    assert ocfg.padded_size == (201, 201, 197)
    solver = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=fb, precision="float64",
                                    max_rhs=1)
    eps = O.phantom_bead(grid, [1.4 ** 2], 20.0, permittivity_bg=eps_bg)
    pot = O.build_potential(ocfg, eps, eps_bg, wl)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, wl)
    x = random_field(ocfg.padded_size + (3,), 41)
    assert rel(plan.green_apply(x), O.green_conv(x, ocfg, pot.k_square)) < 1e-12
    assert rel(plan.apply_operator(x), O.cbs_operator(x, pot.V, ocfg, pot.k_square)) < 1e-12
    solver.release()


def test_general_size_batch_equals_single():
    grid = (15, 12, 10)
    ocfg, solver = configs(grid, absorbing_z(grid[2]), precision="float64")
    pot = O.build_potential(ocfg, bead(grid, 3.0), EPS_BG, WL)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    xs = [random_field(ocfg.padded_size + (3,), s) for s in (51, 52, 53)]
    Y = plan.apply_operator(np.asfortranarray(np.stack(xs, axis=-1)))
    for i, x in enumerate(xs):
        assert np.array_equal(Y[..., i], plan.apply_operator(x))
    solver.release()
