"""The reference's own first example, examples/basic_scattering.jl, end to end on the GPU against the oracle: a
128x128x64 grid at 50 nm, periodic x and y, a 3 um Tanh absorbing layer on z (padded z 124: a non-power-of-two
axis, the general passes with a Bluestein z transform), a SiO2 bead (n = 1.46, radius 10 px) in water, an
x-polarised 532 nm plane wave along +z, GMRES as LinearSolve's KrylovJL_GMRES runs it, tolerance 1e-2.  FP64
follows the oracle to the iteration and to 1e-10; the FP32-storage form stays within 1e-5.
"""
import warnings

import pytest

from _cases import rel
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu

GRID, RES, WL, EPS_BG = (128, 128, 64), (50e-9,) * 3, 532e-9, 1.333 ** 2


@pytest.fixture(scope="module")
def oracle_solution():
    cfg = O.SolverConfig(RES, GRID, (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(3e-6, 3e-6, 1.0)),
                         tolerance=1e-2, method="gmres")
    eps = O.phantom_bead(GRID, [1.46 ** 2], 10.0, permittivity_bg=EPS_BG)
    return O.solve(cfg, O.PlaneWave(WL, [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]), eps, EPS_BG)


@pytest.mark.parametrize("precision,tol", [("float64", 1e-10), ("float32-math64", 1e-5)])
def test_basic_scattering_example(oracle_solution, precision, tol):
    bc_z = F.AbsorbingBoundaryCondition(thickness=3e-6, attenuation_thickness=3e-6, sharpness=1.0,
                                        profile=F.TanhProfile)
    solver = F.ConvergentBornSolver(resolution=RES, grid_size=GRID,
                                    boundary_conditions=(F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(),
                                                         bc_z),
                                    iterations_max=-1, tolerance=1e-2, precision=precision,
                                    linear_solver=F.KrylovJL_GMRES())
    assert solver.padded_size()[2] == 124
    phantom = F.phantom_bead(GRID, [1.46 ** 2], 10.0, permittivity_bg=EPS_BG, on_device=True)
    src = F.PlaneWaveSource(wavelength=WL, polarization=[1.0, 0.0, 0.0], k_vector=[0.0, 0.0, 1.0], amplitude=1.0)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        field = F.solve(solver, src, phantom)
    ref = oracle_solution
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
    assert rel(field.E, ref.E) < tol
    assert rel(field.H, ref.H) < tol
    solver.release()
