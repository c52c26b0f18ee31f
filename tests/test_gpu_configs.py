"""The stated single-RHS configurations against the CPU oracle's FP64 solve (GMRES as the reference runs it:
no restart, MGS, warm start b, maxiters = max(2 Bornmax, 100), tolerance 1e-6; src/solvers/convergent_born.jl:565-600,
703-774).  Periodic x, y and absorbing z with thickness = attenuation thickness = Nz dz, sharpness 1, Tanh.

* Plain CBS, FP64: 64x64x32 at 50 nm, water background (eps 1.33^2), one centred bead of radius 8 px and eps 1.5^2,
  500 nm, x-polarised, +z.  The FP64 plan returns the oracle's iterate within 1e-10 (relative L2 of the cropped E and
  H) after the same number of iterations.
* Precision: 128x128x64, one bead of radius 16 px, otherwise the same.  Complex64 fields -- FP32 arithmetic, and FP32
  storage with FP64 arithmetic, with classical and with block Gram-Schmidt -- stay within 1e-5 of the oracle's FP64
  solve on E and on H; the FP64 plan stays within 1e-10.
"""
import functools
import warnings

import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, bead, configs, rel, xpol
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-5
PLAIN = (64, 64, 32)
PRECISION = (128, 128, 64)


@functools.lru_cache(maxsize=2)
def _oracle(grid):
    ocfg, _ = configs(grid, absorbing_z(grid[2]))
    eps = bead(grid, grid[2] / 4)
    return O.solve(ocfg, xpol()[0], eps, EPS_BG), eps


def _gpu(grid, precision, linear_solver=None):
    _, solver = configs(grid, absorbing_z(grid[2]), precision=precision, linear_solver=linear_solver)
    ref, eps = _oracle(grid)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, xpol()[1], F.Medium(eps, EPS_BG))
    try:
        return out, solver.iteration_count, list(solver.residual_history), ref
    finally:
        solver.release()


def test_plain_fp64_64x64x32_matches_oracle():
    out, iters, hist, ref = _gpu(PLAIN, "float64", F.KrylovJL_GMRES(ortho="mgs"))
    assert ref.potential.Bornmax == 16 and ref.iterations == 100
    assert iters == ref.iterations
    assert hist[-1] == pytest.approx(ref.residuals[-1], rel=1e-8)
    assert rel(out.E, ref.E) < FP64_TOL
    assert rel(out.H, ref.H) < FP64_TOL


@pytest.mark.parametrize("precision,ortho", [("float32", "cgs"), ("float32-math64", "cgs"),
                                             ("float32-math64", "block"), ("float64", "mgs")])
def test_precision_128x128x64_against_oracle(precision, ortho):
    ls = F.KrylovJL_GMRES(ortho=ortho, block_size=8) if ortho == "block" else F.KrylovJL_GMRES(ortho=ortho)
    out, iters, _, ref = _gpu(PRECISION, precision, ls)
    tol = FP64_TOL if precision == "float64" else FP32_TOL
    e, h = rel(out.E, ref.E), rel(out.H, ref.H)
    print(f"precision configuration {precision}/{ortho}: rel-L2 E {e:.3e} H {h:.3e} ({iters} iterations)")
    assert e < tol and h < tol, (e, h)
    if precision == "float64":
        assert iters == ref.iterations
