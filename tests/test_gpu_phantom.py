"""Phantoms painted on the device (fm_phantom_fill) against the CPU oracle's restatement of the reference's
generators (phantoms.jl:58-362), bit for bit, and a solve from a device phantom against the same solve from the
host array."""
import numpy as np
import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, rel
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu


def _plan(grid):
    # painting only needs the unpadded grid: periodic axes keep every size plannable
    solver = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=(F.PeriodicBoundaryCondition(),) * 3,
                                    precision="float64", max_rhs=1)
    return solver, solver.plan()


def _paint(grid, medium):
    solver, plan = _plan(grid)
    try:
        return plan.fill_phantom(medium.shapes, medium.permittivity_bg, copy_out=True)
    finally:
        solver.release()


@pytest.mark.parametrize("grid", [(32, 32, 16), (21, 30, 17), (201, 201, 191)])
def test_device_phantoms_match_oracle(grid):
    cases = [
        (F.phantom_bead(grid, [2.25, 2.0 + 0.05j, 3.0], 4.5, permittivity_bg=1.7, on_device=True),
         O.phantom_bead(grid, [2.25, 2.0 + 0.05j, 3.0], 4.5, permittivity_bg=1.7)),
        (F.phantom_bead(grid, [2.25], 40.0, permittivity_bg=EPS_BG, on_device=True),  # clipped by the grid
         O.phantom_bead(grid, [2.25], 40.0, permittivity_bg=EPS_BG)),
    ]
    for ax in (1, 2, 3):
        cases.append((F.phantom_plate(grid, [2.0], 5, permittivity_bg=1.0, plate_normal=ax, on_device=True),
                      O.phantom_plate(grid, [2.0], 5, permittivity_bg=1.0, plate_normal=ax)))
        cases.append((F.phantom_cylinder(grid, [2.1 + 0.01j], 6.5, permittivity_bg=1.2, height_pixel=9, axis=ax,
                                         on_device=True),
                      O.phantom_cylinder(grid, [2.1 + 0.01j], 6.5, permittivity_bg=1.2, height_pixel=9, axis=ax)))
    for dev, ref in cases:
        assert np.array_equal(_paint(grid, dev), ref)


def test_device_random_beads_and_overlaps_match_host_painting():
    grid = (64, 48, 40)
    med = F.phantom_random_beads(grid, 12, (2, 8), (1.36, 1.60), EPS_BG, 17, on_device=True)
    assert np.array_equal(_paint(grid, med), med.permittivity)
    # overlapping shapes of all kinds in order, centres on half voxels (rounding ties of the bounding boxes)
    shapes = [F.Shape(0, (20.5, 24.0, 20.5), 2.25, radius=10.5), F.Shape(1, (0, 0, 20.5), 1.5, axis=3, extent=3.0),
              F.Shape(2, (32.5, 24.5, 20.0), 3.0 + 0.2j, radius=4.5, axis=2, extent=11.0),
              F.Shape(0, (1.5, 1.5, 1.5), 4.0, radius=2.5)]
    dp = F.DevicePhantom(grid, shapes, EPS_BG)
    assert np.array_equal(_paint(grid, dp), F.paint_host(grid, shapes, EPS_BG))


def test_solve_from_device_phantom_equals_host_array():
    grid = (32, 32, 16)
    dev = F.phantom_random_beads(grid, 3, (2, 5), (1.36, 1.60), EPS_BG, 5, on_device=True)
    host = F.Medium(dev.permittivity, EPS_BG)
    src = F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1])
    out = []
    for med in (dev, host):
        solver = F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=absorbing_z(grid[2])[1],
                                        precision="float64", tolerance=1e-8)
        out.append((F.solve(solver, src, med), solver.iteration_count))
        solver.release()
    (fd, itd), (fh, ith) = out
    assert itd == ith
    assert np.array_equal(fd.E, fh.E) and np.array_equal(fd.H, fh.H)
    # and both against the oracle's solve of the host array
    cfg = O.SolverConfig(RES, grid, absorbing_z(grid[2])[0], tolerance=1e-8, method="gmres")
    ref = O.solve(cfg, O.PlaneWave(WL, [1, 0, 0], [0, 0, 1]), host.permittivity, EPS_BG)
    assert rel(fd.E, ref.E) < 1e-10 and rel(fd.H, ref.H) < 1e-10


def test_build_potential_without_permittivity_needs_a_phantom():
    solver, plan = _plan((16, 16, 8))
    try:
        with pytest.raises(ValueError):
            plan.build_potential(None, EPS_BG, WL, solver.attenuation_filters(), -1)
    finally:
        solver.release()
