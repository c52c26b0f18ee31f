"""Slot engine (fm_engine_*) and the serving loop on the GPU.

Each right-hand side in the engine runs the GMRES iteration of ``solve`` (warm start b, the same stopping
test; restarted every ``basis`` iterations), so:
* a request alone in the engine matches ``solve_batch`` with the same Gram-Schmidt variant and the oracle;
* a request's result is the same alone and admitted in the middle of a mix of other requests, within the
  stated tolerance (FP64 plan 1e-10, FP32 forms 1e-5 relative L2);
* with a basis smaller than the iteration limit it matches GMRES(basis).
"""
import ctypes

import numpy as np
import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, rel
from oracle import cbs_oracle as O

import fmcuda as F
from fmcuda import _lib
from fmcuda import serving as SV

pytestmark = pytest.mark.gpu

SOLVE_TOL = {"float64": 1e-10, "float32": 1e-5, "float32-math64": 1e-5}
GRID = (32, 32, 16)


def _request(req_id, seed, nsrc, grid=GRID, tol=1e-6):
    med = F.phantom_random_beads(grid, 3, (2, 5), (1.36, 1.60), EPS_BG, seed)
    cone = F.illumination_cone(grid, RES, WL, EPS_BG, nsrc, 1.2, seed)
    return SV.Request(req_id=req_id, medium=med, sources=cone[:nsrc], tolerance=tol)


def _solver(precision, grid=GRID, tol=1e-6, restart=0, max_rhs=8):
    return F.ConvergentBornSolver(resolution=RES, grid_size=grid, boundary_conditions=absorbing_z(grid[2])[1],
                                  tolerance=tol, precision=precision, max_rhs=max_rhs,
                                  linear_solver=F.KrylovJL_GMRES(ortho="cgs", gmres_restart=restart))


def _batch_reference(req, precision, restart=0):
    solver = _solver(precision, req.shape, req.tolerance, restart)
    out = F.solve_batch(solver, [[s] for s in req.sources], req.medium)
    info = solver.last_info
    solver.release()
    return out, info


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_engine_alone_matches_solve_batch_and_oracle(precision):
    req = _request(1, 11, 3)
    eng = SV.Engine(_solver(precision), slots=4, basis=100, wavelength=WL, permittivity_bg=EPS_BG)
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
    # one right-hand side against the oracle (Krylov.jl semantics, FP64 numpy)
    ocfg = O.SolverConfig(RES, GRID, absorbing_z(GRID[2])[0], tolerance=req.tolerance, method="gmres")
    s = req.sources[0]
    oref = O.solve(ocfg, O.PlaneWave(WL, s.polarization, s.k_vector), req.medium.permittivity, EPS_BG)
    assert rel(req.E[..., 0], oref.E) < SOLVE_TOL[precision]
    assert rel(req.H[..., 0], oref.H) < SOLVE_TOL[precision]


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_engine_result_same_alone_and_in_mix(precision):
    """Request A alone, then A admitted while B runs and before C arrives, with fewer slots than
    right-hand sides (so admission waits for slots to free up)."""
    a_alone = _request(0, 21, 2)
    eng = SV.Engine(_solver(precision), slots=3, basis=100, wavelength=WL, permittivity_bg=EPS_BG)
    try:
        eng.submit(a_alone)
        eng.drain([a_alone])
        a_mix, b, c = _request(1, 21, 2), _request(2, 22, 3), _request(3, 23, 1)
        eng.submit(b)
        for _ in range(2):
            for rid, rhs, info in eng.step():
                eng.complete(rid, rhs, info)
        eng.submit(a_mix)
        for _ in range(5):
            for rid, rhs, info in eng.step():
                eng.complete(rid, rhs, info)
        eng.submit(c)
        eng.drain([a_mix, b, c])
        assert eng.status() == (0, 0)
    finally:
        eng.close()
    for k in range(2):
        assert rel(a_mix.E[..., k], a_alone.E[..., k]) < SOLVE_TOL[precision]
        assert rel(a_mix.H[..., k], a_alone.H[..., k]) < SOLVE_TOL[precision]
        assert a_mix.infos[k]["iterations"] == a_alone.infos[k]["iterations"]
    # the other members of the mix are right too
    for r in (b, c):
        ref, _ = _batch_reference(r, precision)
        for k in range(len(r.sources)):
            assert rel(r.E[..., k], ref[k].E) < SOLVE_TOL[precision]


def test_engine_restart_matches_gmres_restart():
    """basis 8 < iteration limit: the engine restarts like GMRES(8)."""
    req = _request(5, 31, 2)
    eng = SV.Engine(_solver("float64"), slots=2, basis=8, wavelength=WL, permittivity_bg=EPS_BG)
    try:
        eng.submit(req)
        eng.drain([req])
    finally:
        eng.close()
    ref, info = _batch_reference(req, "float64", restart=8)
    for b in range(2):
        assert req.infos[b]["iterations"] == info[b]["iterations"]
        assert req.infos[b]["iterations"] > 8
        assert rel(req.E[..., b], ref[b].E) < 1e-10
        assert rel(req.H[..., b], ref[b].H) < 1e-10


def test_engine_rejects_bad_requests():
    eng = SV.Engine(_solver("float32-math64"), slots=1, basis=20, wavelength=WL, permittivity_bg=EPS_BG)
    try:
        req = _request(9, 41, 1)
        req.sources[0].wavelength = 600e-9
        with pytest.raises(ValueError):
            eng.submit(req)
        req = _request(10, 41, 1)
        req.medium.permittivity[0, 0, 0] = np.nan
        with pytest.raises(_lib.FMError):
            eng.submit(req)
        g = GRID
        w = (_lib.fm_plane_wave * 1)()
        w[0].wavelength = WL
        w[0].polarization[0] = 0.0
        w[0].polarization[4] = 1.0          # along k: not transverse
        w[0].k_vector[2] = 1.0
        w[0].amplitude = 1.0
        eps = np.full(g, EPS_BG, dtype=np.complex128, order="F")
        E = np.empty(g + (3,), dtype=np.complex128, order="F")
        st = _lib.lib().fm_engine_submit(eng.handle, 1, _lib.ptr(eps), 1, w, 1e-5, -1, _lib.ptr(E), _lib.ptr(E))
        assert st == _lib.FM_ERR_INVALID
        assert eng.status() == (0, 0)
    finally:
        eng.close()


def test_server_mixed_shapes_latency_and_results():
    shapes = ((32, 32, 16), (64, 32, 32))
    reqs = SV.serving_requests(8, rate=200.0, shapes=shapes, max_angles=4, seed=3, beads=3, radius_range=(2, 5))
    with SV.Server(shapes, budget_bytes=4e9, basis=100, slots={shapes[0]: 4, shapes[1]: 3}) as srv:
        rep = SV.run_stream(srv, reqs, timeout=600)
    assert rep["requests"] == 8 and rep["solves"] == sum(len(r.sources) for r in reqs)
    assert 0 < rep["p50_latency_s"] <= rep["p99_latency_s"]
    for r in reqs[:4]:
        ref, _ = _batch_reference(r, "float32-math64")
        for k in range(len(r.sources)):
            assert rel(r.E[..., k], ref[k].E) < 1e-5
            assert rel(r.H[..., k], ref[k].H) < 1e-5
