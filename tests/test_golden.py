"""Committed golden fixtures (tests/golden, made by make_golden.py from the oracle).

CPU: the oracle still reproduces them.  GPU: libfmcuda (through the C ABI) matches them."""
import os
import warnings

import numpy as np
import pytest

from oracle import cbs_oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RES = (50e-9,) * 3
EPS_BG = 1.33 ** 2
WL = 500e-9


def _load(name):
    return np.load(os.path.join(HERE, name))


def _solve_cfg():
    g = (16, 16, 8)
    bz = O.AbsorbingBC(g[2] * RES[2], g[2] * RES[2], 1.0)
    return O.SolverConfig(RES, g, (O.PeriodicBC(), O.PeriodicBC(), bz), tolerance=1e-6)


def test_oracle_reproduces_solve_fixture():
    d = _load("solve_16x16x8_bead.npz")
    r = O.solve(_solve_cfg(), O.PlaneWave(WL, [1, 0, 0], [0, 0, 1]), d["eps"], EPS_BG)
    assert r.iterations == int(d["iterations"])
    assert O.rel_l2(r.E, d["E"]) < 1e-12 and O.rel_l2(r.H, d["H"]) < 1e-12


def test_oracle_reproduces_green_fixture():
    d = _load("green_8x16x8.npz")
    g = (8, 16, 8)
    bz = O.AbsorbingBC(g[2] * RES[2], g[2] * RES[2], 1.0)
    cfg = O.SolverConfig(RES, g, (O.PeriodicBC(), O.PeriodicBC(), bz))
    pot = O.build_potential(cfg, d["eps"], EPS_BG, WL)
    assert O.rel_l2(pot.V, d["V"]) < 1e-15
    assert O.rel_l2(O.green_conv(d["x"], cfg, pot.k_square), d["green"]) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("float64", 1e-10), ("float32", 1e-5), ("float32-math64", 1e-5)])
def test_library_matches_solve_fixture(precision, tol):
    import fmcuda as F
    d = _load("solve_16x16x8_bead.npz")
    bz = F.AbsorbingBoundaryCondition(thickness=8 * RES[2], attenuation_thickness=8 * RES[2], sharpness=1.0)
    s = F.ConvergentBornSolver(resolution=RES, grid_size=(16, 16, 8),
                               boundary_conditions=(F.PeriodicBoundaryCondition(),) * 2 + (bz,), precision=precision,
                               linear_solver=F.KrylovJL_GMRES(ortho="mgs"))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(s, F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1]),
                      F.Medium(d["eps"], EPS_BG))
    assert O.rel_l2(out.E, d["E"]) < tol and O.rel_l2(out.H, d["H"]) < tol
    if precision == "float64":
        assert s.iteration_count == int(d["iterations"])
        assert s.residual_history[-1] == pytest.approx(float(d["residuals"][-1]), rel=1e-8)


@pytest.mark.gpu
def test_library_matches_green_fixture():
    import fmcuda as F
    d = _load("green_8x16x8.npz")
    bz = F.AbsorbingBoundaryCondition(thickness=8 * RES[2], attenuation_thickness=8 * RES[2], sharpness=1.0)
    s = F.ConvergentBornSolver(resolution=RES, grid_size=(8, 16, 8),
                               boundary_conditions=(F.PeriodicBoundaryCondition(),) * 2 + (bz,), precision="float64")
    p = s.plan()
    p.set_potential(d["V"], float(d["k_bg"]), float(d["eps_imag"]), WL)
    assert O.rel_l2(p.green_apply(d["x"]), d["green"]) < 1e-12
    assert O.rel_l2(p.apply_operator(d["x"]), d["op"]) < 1e-12
