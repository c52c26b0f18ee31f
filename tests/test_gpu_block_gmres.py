"""s-step (block) GMRES on the GPU (FM_ORTHO_BLOCK) against the oracle's GMRES (Krylov.jl semantics, MGS).

In exact arithmetic block GMRES takes the same iterates as full GMRES, so the bars are those of the
other solve tests: FP64 plan <= 1e-10 relative L2 with the same iteration count, FP32 forms <= 1e-5.
"""
import warnings

import numpy as np
import pytest

from _cases import EPS_BG, WL, absorbing_z, bead, configs, rel, xpol
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu

SOLVE_TOL = {"float64": 1e-10, "float32": 1e-5, "float32-math64": 1e-5}


def _solve(grid, radius, precision, block, tol=1e-6, sources=None, store="fp64"):
    ls = F.KrylovJL_GMRES(ortho="block", block_size=block, block_vectors=store)
    ocfg, solver = configs(grid, absorbing_z(grid[2]), tol=tol, precision=precision, linear_solver=ls)
    eps = bead(grid, radius)
    osrc, fsrc = sources if sources is not None else xpol()
    ref = O.solve(ocfg, osrc, eps, EPS_BG)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, fsrc, F.Medium(eps, EPS_BG))
    return ref, out, solver


@pytest.mark.parametrize("precision,block", [("float64", 2), ("float64", 3), ("float64", 4), ("float64", 5),
                                             ("float64", 6), ("float64", 8), ("float64", 16), ("float32-math64", 3),
                                             ("float32-math64", 4), ("float32-math64", 5), ("float32-math64", 6),
                                             ("float32", 4)])
def test_block_gmres_matches_oracle(precision, block):
    """100 non-converged iterations (the reference's iteration limit on this case)."""
    ref, out, solver = _solve((32, 32, 16), 4.0, precision, block)
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
        assert abs(solver.residual_history[-1] - ref.residual) <= 1e-8 * ref.residual
    assert rel(out.E, ref.E) < SOLVE_TOL[precision]
    assert rel(out.H, ref.H) < SOLVE_TOL[precision]


@pytest.mark.parametrize("block", [3, 4])
def test_block_gmres_stops_inside_a_block(block):
    """A loose tolerance makes GMRES stop after a few iterations, in the middle of a block: the stopping
    iteration and the iterate must be those of full GMRES."""
    ref, out, solver = _solve((16, 16, 8), 2.0, "float64", block, tol=1e-3)
    assert ref.solved and ref.iterations < 30
    assert solver.iteration_count == ref.iterations
    assert solver.last_info[0]["solved"]
    assert rel(out.E, ref.E) < 1e-10


def test_block_gmres_batch_equals_single():
    grid = (16, 16, 8)
    ls = F.KrylovJL_GMRES(ortho="block", block_size=4)
    ocfg, solver = configs(grid, absorbing_z(8), precision="float64", linear_solver=ls)
    med = F.Medium(bead(grid, 3.0), EPS_BG)
    srcs = [F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1]),
            F.PlaneWaveSource(wavelength=WL, polarization=[0, 1, 0], k_vector=[0.6, 0, 0.8]),
            F.PlaneWaveSource(wavelength=WL, polarization=[0, 1, 0], k_vector=[0, 0, 1])]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        outs = F.solve_batch(solver, srcs, med)
        for s, o in zip(srcs, outs):
            one = F.solve(solver, s, med)
            assert rel(o.E, one.E) < 1e-12
            assert rel(o.H, one.H) < 1e-12


@pytest.mark.parametrize("store", ["fp64", "storage", "fp64-ortho"])
def test_block_gmres_oblique_fp32_math64(store):
    """Both kinds of raw block vectors on the FP32-storage / FP64-arithmetic plan."""
    grid = (32, 32, 16)
    src = F.illumination_cone(grid, (50e-9,) * 3, WL, EPS_BG, 4, 1.2, 11)[3]
    pair = (O.PlaneWave(WL, src.polarization, src.k_vector), src)
    ref, out, _ = _solve(grid, 5.0, "float32-math64", 4, sources=pair, store=store)
    assert rel(out.E, ref.E) < 1e-5
    assert rel(out.H, ref.H) < 1e-5


def test_block_gmres_rejects_restart_and_bad_sizes():
    grid = (16, 16, 8)
    for ls in (F.KrylovJL_GMRES(ortho="block", gmres_restart=10), F.KrylovJL_GMRES(ortho="block", block_size=9),
               F.KrylovJL_GMRES(ortho="block", block_size=17)):
        ocfg, solver = configs(grid, absorbing_z(8), linear_solver=ls)
        with pytest.raises((ValueError, F._lib.FMError)):
            F.solve(solver, xpol()[1], F.Medium(bead(grid, 2.0), EPS_BG))


@pytest.mark.parametrize("precision,block", [("float64", 4), ("float64", 7), ("float32-math64", 4),
                                             ("float32", 3)])
def test_bulk_block_dot_matches_register_block_dot(precision, block):
    """The bulk-copy pipelined block dot (one CTA per SM over all active right-hand sides) against the
    register-staged one, on a batch whose right-hand sides stop at different iterations, so the list of
    active right-hand sides changes during the solve."""
    from fmcuda import autotune as AT
    grid = (16, 16, 8)
    ls = F.KrylovJL_GMRES(ortho="block", block_size=block)
    ocfg, solver = configs(grid, absorbing_z(8), tol=1e-4, precision=precision, linear_solver=ls)
    med = F.Medium(bead(grid, 3.0), EPS_BG)
    srcs = [F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1]),
            F.PlaneWaveSource(wavelength=WL, polarization=[0, 1, 0], k_vector=[0.6, 0, 0.8]),
            F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0.8, 0.6])]
    res = {}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        for bulk in (1, 0):
            AT.apply(solver.plan(), {"block_dot": bulk})
            outs = F.solve_batch(solver, srcs, med)
            res[bulk] = (outs, [i["iterations"] for i in solver.last_info])
    AT.apply(solver.plan(), {"block_dot": AT.DEFAULT["block_dot"]})
    tol = 1e-10 if precision == "float64" else 1e-5
    assert len(set(res[1][1])) > 1, "right-hand sides should stop at different iterations"
    if precision == "float64":
        assert res[1][1] == res[0][1]
    for a, b in zip(res[1][0], res[0][0]):
        assert rel(a.E, b.E) < tol
        assert rel(a.H, b.H) < tol
    solver.release()


@pytest.mark.parametrize("precision,block", [("float64", 4), ("float64", 8), ("float64", 16), ("float32-math64", 4),
                                             ("float32-math64", 8), ("float32-math64", 16)])
def test_block_gmres_orthonormal_block_storage(precision, block):
    """Blocks stored orthonormalised (V = Y' Rb^{-1}) take the iterates of full GMRES like raw storage."""
    ref, out, solver = _solve((32, 32, 16), 4.0, precision, block, store="fp64-ortho")
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
        assert abs(solver.residual_history[-1] - ref.residual) <= 1e-8 * ref.residual
    assert rel(out.E, ref.E) < SOLVE_TOL[precision]
    assert rel(out.H, ref.H) < SOLVE_TOL[precision]


def test_block_gmres_orthonormal_storage_stops_inside_a_block():
    ref, out, solver = _solve((16, 16, 8), 2.0, "float64", 4, tol=1e-3, store="fp64-ortho")
    assert ref.solved and ref.iterations < 30
    assert solver.iteration_count == ref.iterations
    assert rel(out.E, ref.E) < 1e-10
