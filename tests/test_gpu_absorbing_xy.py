"""Absorbing boundaries on x and y: sub-pixel shifts of 1/4 on every absorbing axis
(src/solvers/boundary_conditions.jl:518-527), phase ramps over all three axes (src/core/dyadic_green.jl:243-266),
and the average of the +s and -s branches (dyadic_green.jl:127-152).  The library runs the two branches as two
sweeps of the five axis passes; these tests compare it with the CPU oracle.

Tolerances as in the other parity tests: FP64 <= 1e-12 for single applications and <= 1e-10 for solves
(with the oracle's iteration count); FP32 forms 2e-6 / 2e-7 for single applications and 1e-5 for solves.
"""
import warnings

import pytest

from _cases import EPS_BG, RES, WL, bead, configs, random_field, rel, xpol
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu

OP_TOL = {"float64": 1e-12, "float32": 2e-6, "float32-math64": 2e-7}
SOLVE_TOL = {"float64": 1e-10, "float32": 1e-5, "float32-math64": 1e-5}


def absorbing_on(grid, axes):
    """Absorbing (thickness = attenuation thickness = N_d dd, sharpness 1, Tanh) on ``axes``, periodic elsewhere."""
    ob, fb = [], []
    for d in range(3):
        if d in axes:
            t = grid[d] * RES[d]
            ob.append(O.AbsorbingBC(t, t, 1.0, O.TANH))
            fb.append(F.AbsorbingBoundaryCondition(thickness=t, attenuation_thickness=t, sharpness=1.0,
                                                   profile=F.TanhProfile))
        else:
            ob.append(O.PeriodicBC())
            fb.append(F.PeriodicBoundaryCondition())
    return tuple(ob), tuple(fb)


CASES = [((16, 16, 8), (0, 1, 2)), ((16, 32, 16), (0,)), ((32, 16, 16), (1,)), ((16, 16, 16), (0, 2))]


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
@pytest.mark.parametrize("grid,axes", CASES)
def test_green_and_operator_absorbing_xy(precision, grid, axes):
    ocfg, solver = configs(grid, absorbing_on(grid, axes), precision=precision)
    eps = bead(grid, min(grid) / 4)
    pot = O.build_potential(ocfg, eps, EPS_BG, WL)
    assert all(ocfg.shifts[d] == (0.25 if d in axes else 0.0) for d in range(3))
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    x = random_field(ocfg.padded_size + (3,), 21)
    assert rel(plan.green_apply(x), O.green_conv(x, ocfg, pot.k_square)) < OP_TOL[precision]
    y0 = random_field(ocfg.padded_size + (3,), 22)
    a, b = 0.6 + 0.3j, -0.4 + 1.1j
    ref = O.cbs_operator(x, pot.V, ocfg, pot.k_square, alpha=a, beta=b, y=y0)
    assert rel(plan.apply_operator(x, y0, alpha=a, beta=b), ref) < OP_TOL[precision]
    solver.release()


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
@pytest.mark.parametrize("grid,axes", [((16, 16, 8), (0, 1, 2)), ((16, 32, 16), (0,))])
def test_solve_absorbing_xy(precision, grid, axes):
    ocfg, solver = configs(grid, absorbing_on(grid, axes), precision=precision,
                           linear_solver=F.KrylovJL_GMRES(ortho="mgs" if precision == "float64" else "cgs"))
    eps = bead(grid, 3.0)
    osrc, fsrc = xpol()
    ref = O.solve(ocfg, osrc, eps, EPS_BG)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, fsrc, F.Medium(eps, EPS_BG))
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
    assert rel(out.E, ref.E) < SOLVE_TOL[precision]
    assert rel(out.H, ref.H) < SOLVE_TOL[precision]
    solver.release()


def test_block_gmres_absorbing_all_axes_fp64():
    """Block (s-step) GMRES takes full GMRES's iterate with the two-branch operator too."""
    grid = (16, 16, 8)
    ocfg, solver = configs(grid, absorbing_on(grid, (0, 1, 2)), precision="float64",
                           linear_solver=F.KrylovJL_GMRES(ortho="block", block_size=4))
    eps = bead(grid, 3.0)
    osrc, fsrc = xpol()
    ref = O.solve(ocfg, osrc, eps, EPS_BG)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, fsrc, F.Medium(eps, EPS_BG))
    assert solver.iteration_count == ref.iterations
    assert rel(out.E, ref.E) < 1e-10 and rel(out.H, ref.H) < 1e-10
    solver.release()
