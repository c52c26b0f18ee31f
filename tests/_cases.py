"""Shared test scenarios: the same configuration expressed for the oracle and for fmcuda."""
import numpy as np

from oracle import cbs_oracle as O

import fmcuda as F

RES = (50e-9, 50e-9, 50e-9)
EPS_BG = 1.33 ** 2
WL = 500e-9


def absorbing_z(nz, res=RES[2]):
    """Periodic x, y; absorbing z with thickness = attenuation_thickness = Nz*dz, sharpness 1, Tanh."""
    t = nz * res
    return ((O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(t, t, 1.0, O.TANH)),
            (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(),
             F.AbsorbingBoundaryCondition(thickness=t, attenuation_thickness=t, sharpness=1.0,
                                          profile=F.TanhProfile)))


def periodic():
    return ((O.PeriodicBC(),) * 3, (F.PeriodicBoundaryCondition(),) * 3)


def configs(grid, bcs_pair, tol=1e-6, precision="float64", linear_solver=None, method="gmres"):
    ob, fb = bcs_pair
    ocfg = O.SolverConfig(RES, grid, ob, tolerance=tol, method=method)
    solver = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=fb, tolerance=tol,
                                    precision=precision, linear_solver=linear_solver, max_rhs=8)
    return ocfg, solver


def bead(grid, radius, eps=2.25):
    return O.phantom_bead(grid, [eps], radius, permittivity_bg=EPS_BG)


def random_field(shape, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def xpol():
    return O.PlaneWave(WL, [1, 0, 0], [0, 0, 1]), F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0],
                                                                     k_vector=[0, 0, 1])


def rel(a, b):
    return O.rel_l2(a, b)
