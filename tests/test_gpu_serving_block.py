"""Slot engine with block GMRES (fm_engine_create with FM_ORTHO_BLOCK) on the GPU.

A slot whose iteration limit fits the basis runs the batched s-step block GMRES (s = 8, FP64 block vectors
stored orthonormalised): its first 8 iterations share the engine's CGS launches, then every engine step
advances it by one block, in launches shared with the other block slots, each at its own basis size.  So:
* a request alone in a block engine matches ``solve_batch`` with ``ortho="block"`` (same iteration count on
  the FP64 plan) and the oracle;
* its result is the same alone and admitted into a mix whose slots sit at other iterations;
* a slot whose limit does not fit the basis restarts when the basis is full, every floor(basis / 8) * 8
  iterations, and matches GMRES with that restart length.
"""
import numpy as np
import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, rel
from oracle import cbs_oracle as O

import fmcuda as F
from fmcuda import _lib
from fmcuda import serving as SV

pytestmark = pytest.mark.gpu

SOLVE_TOL = {"float64": 1e-10, "float32-math64": 1e-5}
GRID = (32, 32, 16)
BASIS = 112  # >= 100 iterations + 8 block vectors


def _request(req_id, seed, nsrc, grid=GRID, tol=1e-6):
    med = F.phantom_random_beads(grid, 3, (2, 5), (1.36, 1.60), EPS_BG, seed)
    cone = F.illumination_cone(grid, RES, WL, EPS_BG, nsrc, 1.2, seed)
    return SV.Request(req_id=req_id, medium=med, sources=cone[:nsrc], tolerance=tol)


def _solver(precision, grid=GRID, tol=1e-6, ortho="block", restart=0, iterations_max=-1, max_rhs=8):
    return F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=absorbing_z(grid[2])[1],
                                  tolerance=tol, precision=precision, max_rhs=max_rhs, iterations_max=iterations_max,
                                  linear_solver=F.KrylovJL_GMRES(ortho=ortho, gmres_restart=restart,
                                                                 block_size=8, block_vectors="fp64-ortho"))


def _batch_reference(req, precision, **kw):
    solver = _solver(precision, req.shape, req.tolerance, **kw)
    out = F.solve_batch(solver, [[s] for s in req.sources], req.medium)
    info = solver.last_info
    solver.release()
    return out, info


def _step(eng, n):
    for _ in range(n):
        for rid, rhs, info in eng.step():
            eng.complete(rid, rhs, info)


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_block_engine_alone_matches_block_solve_and_oracle(precision):
    req = _request(1, 11, 3)
    eng = SV.Engine(_solver(precision), slots=4, basis=BASIS, wavelength=WL, permittivity_bg=EPS_BG, ortho="block")
    try:
        eng.submit(req)
        eng.drain([req])
    finally:
        eng.close()
    ref, info = _batch_reference(req, precision)
    for b in range(3):
        assert rel(req.E[..., b], ref[b].E) < SOLVE_TOL[precision]
        assert rel(req.H[..., b], ref[b].H) < SOLVE_TOL[precision]
        if precision == "float64":
            assert req.infos[b]["iterations"] == info[b]["iterations"]
            assert req.infos[b]["solved"] == info[b]["solved"]
    assert max(i["iterations"] for i in req.infos.values()) > 8  # the block phase ran
    ocfg = O.SolverConfig(RES, GRID, absorbing_z(GRID[2])[0], tolerance=req.tolerance, method="gmres")
    s = req.sources[0]
    oref = O.solve(ocfg, O.PlaneWave(WL, s.polarization, s.k_vector), req.medium.permittivity, EPS_BG)
    assert rel(req.E[..., 0], oref.E) < SOLVE_TOL[precision]
    assert rel(req.H[..., 0], oref.H) < SOLVE_TOL[precision]


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_block_engine_same_alone_and_in_mix_with_cgs_slot(precision):
    """A alone, then A admitted while B runs, next to C whose limit (120 iterations) does not fit the basis
    (C restarts after 112 iterations, as GMRES(112)); fewer slots than right-hand sides."""
    a_alone = _request(0, 21, 2)
    eng = SV.Engine(_solver(precision), slots=3, basis=BASIS, wavelength=WL, permittivity_bg=EPS_BG, ortho="block")
    try:
        eng.submit(a_alone)
        eng.drain([a_alone])
        a_mix, b, c = _request(1, 21, 2), _request(2, 22, 3), _request(3, 23, 1, tol=1e-9)
        eng.submit(b)
        _step(eng, 3)
        eng.submit(c, iterations_max=60)
        _step(eng, 2)
        eng.submit(a_mix)
        eng.drain([a_mix, b, c])
        assert eng.status() == (0, 0)
    finally:
        eng.close()
    for k in range(2):
        assert rel(a_mix.E[..., k], a_alone.E[..., k]) < SOLVE_TOL[precision]
        assert rel(a_mix.H[..., k], a_alone.H[..., k]) < SOLVE_TOL[precision]
        assert a_mix.infos[k]["iterations"] == a_alone.infos[k]["iterations"]
    ref, _ = _batch_reference(b, precision)
    for k in range(3):
        assert rel(b.E[..., k], ref[k].E) < SOLVE_TOL[precision]
        assert rel(b.H[..., k], ref[k].H) < SOLVE_TOL[precision]
    ref, info = _batch_reference(c, precision, ortho="cgs", restart=BASIS, iterations_max=60)
    assert rel(c.E[..., 0], ref[0].E) < SOLVE_TOL[precision]
    assert rel(c.H[..., 0], ref[0].H) < SOLVE_TOL[precision]
    if precision == "float64":
        assert c.infos[0]["iterations"] == info[0]["iterations"]


def test_block_engine_restarts_like_gmres_restart():
    """basis 24 < iteration limit: block cycles of 24 iterations (8 CGS steps and two blocks), as GMRES(24)."""
    req = _request(5, 31, 2)
    eng = SV.Engine(_solver("float64"), slots=2, basis=24, wavelength=WL, permittivity_bg=EPS_BG, ortho="block")
    try:
        eng.submit(req)
        eng.drain([req])
    finally:
        eng.close()
    ref, info = _batch_reference(req, "float64", ortho="cgs", restart=24)
    for b in range(2):
        assert req.infos[b]["iterations"] == info[b]["iterations"]
        assert req.infos[b]["iterations"] > 24
        assert rel(req.E[..., b], ref[b].E) < 1e-10
        assert rel(req.H[..., b], ref[b].H) < 1e-10


@pytest.mark.parametrize("grid", [(15, 12, 10), (15, 13, 9)])
def test_block_engine_on_general_grids(grid):
    """Odd and non-power-of-two axes (the general passes).  On 15x12x10 (3 x padded voxels a multiple of 4) the
    slots run block GMRES; on 15x13x9 they cannot and run CGS in the same block engine.  Either way the engine
    matches the batched solve of the same method on the FP64 plan."""
    med = F.phantom_random_beads(grid, 2, (1.5, 3.0), (1.36, 1.60), EPS_BG, 41)
    cone = F.illumination_cone(grid, RES, WL, EPS_BG, 2, 1.2, 41)
    req = SV.Request(req_id=7, medium=med, sources=cone[:2], tolerance=1e-6)
    eng = SV.Engine(_solver("float64", grid), slots=2, basis=BASIS, wavelength=WL, permittivity_bg=EPS_BG,
                    ortho="block")
    try:
        eng.submit(req)
        eng.drain([req])
    finally:
        eng.close()
    n = int(np.prod(_solver("float64", grid).padded_size()))
    ortho = "block" if (3 * n) % 4 == 0 else "cgs"
    ref, info = _batch_reference(req, "float64", ortho=ortho)
    for b in range(2):
        assert req.infos[b]["iterations"] == info[b]["iterations"]
        assert rel(req.E[..., b], ref[b].E) < 1e-10
        assert rel(req.H[..., b], ref[b].H) < 1e-10
