"""The large configuration's accuracy bar at reduced lateral size (the full 512^3 FP64 solve needs about 182 GB).

128x128x256 at 50 nm with the large configuration's absorbing z (thickness = attenuation thickness = Nz * 50 nm,
padded z 512, the two shifted z branches as two z passes), ten beads with its statistics (radius U[6,24] px,
index U[1.4,2.0]), x-polarised +z illumination, GMRES(20) to the iteration limit: the FP32-storage / FP64-arithmetic
form stays within 1e-5 of the plain FP64 method (MGS, which the oracle pins on smaller grids), E and H, and takes
the same number of iterations.
"""
import warnings

import pytest

from _cases import EPS_BG, RES, WL, rel

import fmcuda as F

pytestmark = pytest.mark.gpu


def test_large_configuration_fp32_form_within_bar_at_padded_z_512():
    grid = (128, 128, 256)
    med = F.phantom_random_beads(grid, 10, (6, 24), (1.4, 2.0), EPS_BG, 20261208)  # the bench check's seed
    bc_z = F.AbsorbingBoundaryCondition(thickness=grid[2] * RES[2], attenuation_thickness=grid[2] * RES[2],
                                        sharpness=1.0, profile=F.TanhProfile)
    bcs = (F.PeriodicBoundaryCondition(), F.PeriodicBoundaryCondition(), bc_z)
    src = F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1])
    out = {}
    for prec, ortho in (("float32-math64", "cgs"), ("float64", "mgs")):
        sv = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=bcs, tolerance=1e-6,
                                    precision=prec, max_rhs=1,
                                    linear_solver=F.KrylovJL_GMRES(ortho=ortho, gmres_restart=20))
        assert sv.padded_size()[2] == 512
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            f = F.solve(sv, src, med)
        out[prec] = (f, sv.iteration_count)
        sv.release()
    (f32, it32), (f64, it64) = out["float32-math64"], out["float64"]
    assert it32 == it64
    assert rel(f32.E, f64.E) < 1e-5
    assert rel(f32.H, f64.H) < 1e-5
