"""The reference's own example, examples/two_beam_interference.jl (test_two_beam_interference_homogeneous), end
to end on the GPU: a 201x201x191 grid at 50 nm (odd axes: the general passes with Bluestein transforms), periodic
x and y, a 300 nm Tanh absorbing layer on z, water (n = 1.333), two coherent x-polarised 532 nm plane waves at
the +-3rd illumination order, BiCGStab as the example runs it, FP64.  The example's own acceptance checks must hold:
fringe contrast >= 0.8 on the central y profile, 2 * 3 fringes (+-2), and 1e-3 < max|E| < 1e3.  In this
homogeneous medium the total field is the coherent sum of the two incident waves, which the oracle computes.
"""
import math
import warnings

import numpy as np
import pytest

from _cases import rel
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu


def _count_maxima(profile):
    """count_intensity_maxima of the example: interior strict local maxima above 10 % of the maximum."""
    top = profile.max()
    return sum(1 for i in range(1, len(profile) - 1)
               if profile[i] > profile[i - 1] and profile[i] > profile[i + 1] and profile[i] > 0.1 * top)


def test_two_beam_interference_homogeneous_example():
    grid, res = (201, 201, 191), (50e-9,) * 3
    bc_z = F.AbsorbingBoundaryCondition(thickness=300e-9, attenuation_thickness=300e-9, sharpness=1.0,
                                        profile=F.TanhProfile)
    solver = F.ConvergentBornSolver(resolution=res, grid_size=grid,
                                    boundary_conditions=(F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(),
                                                         bc_z),
                                    iterations_max=-1, tolerance=1e-6, precision="float64",
                                    linear_solver=F.KrylovJL_BICGSTAB())
    eps_bg = 1.333 ** 2
    wl = 532e-9
    k_bg = 2 * math.pi * math.sqrt(eps_bg) / wl
    ky = 2 * math.pi * 3 / (grid[1] * res[1])
    angle = math.asin(ky / k_bg)
    k1, k2 = [0.0, math.sin(angle), math.cos(angle)], [0.0, -math.sin(angle), math.cos(angle)]
    sources = [F.PlaneWaveSource(wavelength=wl, polarization=[1.0, 0.0, 0.0], k_vector=k1, amplitude=1.0),
               F.PlaneWaveSource(wavelength=wl, polarization=[1.0, 0.0, 0.0], k_vector=k2, amplitude=1.0)]
    medium = F.Medium(np.full(grid, eps_bg, dtype=np.complex128), eps_bg)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        field = F.solve(solver, sources, medium)
    solver.release()

    intensity = np.sum(np.abs(field.E) ** 2, axis=3)
    cx, cz = grid[0] // 2, grid[2] // 2  # div(N, 2) + 1 in 1-based indices
    prof = intensity[cx, :, cz]
    contrast = (prof.max() - prof.min()) / (prof.max() + prof.min())
    assert contrast >= 0.8
    assert abs(_count_maxima(prof) - 6) <= 2
    e_max = np.abs(field.E).max()
    assert 1e-3 < e_max < 1e3

    # the coherent sum of the incident waves on the cropped grid (generate_incident_field, plane_wave.jl:198-268)
    cfg = O.SolverConfig(res, grid, (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(300e-9, 300e-9, 1.0)))
    E_inc = None
    for k in (k1, k2):
        Ei, _ = O.incident_field(O.PlaneWave(wl, [1.0, 0.0, 0.0], k), cfg, eps_bg)
        E_inc = Ei if E_inc is None else E_inc + Ei
    assert rel(field.E, cfg.crop(E_inc)) < 1e-4
