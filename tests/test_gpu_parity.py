"""GPU parity of libfmcuda against the CPU oracle (called through the C ABI via fmcuda).

Tolerances: FP64 plan <= 1e-10 relative L2 (1e-12 for single operator applications);
FP32 plan <= 1e-5 relative L2 (2e-6 for single operator applications).
"""
import warnings

import numpy as np
import pytest

from _cases import EPS_BG, RES, WL, absorbing_z, bead, configs, periodic, random_field, rel, xpol
from oracle import cbs_oracle as O

import fmcuda as F

pytestmark = pytest.mark.gpu

OP_TOL = {"float64": 1e-12, "float32": 2e-6, "float32-math64": 2e-7}
SOLVE_TOL = {"float64": 1e-10, "float32": 1e-5, "float32-math64": 1e-5}


def _plan_with_oracle_potential(grid, bcs, precision):
    ocfg, solver = configs(grid, bcs, precision=precision)
    eps = bead(grid, min(grid) / 4)
    pot = O.build_potential(ocfg, eps, EPS_BG, WL)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    return ocfg, solver, plan, pot


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
@pytest.mark.parametrize("grid,kind", [((32, 32, 16), "absz"), ((16, 32, 8), "absz"), ((32, 16, 32), "per"),
                                       ((64, 32, 32), "absz"), ((96, 32, 16), "absz"), ((32, 96, 16), "absz"),
                                       ((16, 32, 96), "per"), ((16, 16, 128), "absz"), ((16, 8, 512), "per"),
                                       ((8, 16, 256), "absz"), ((8, 512, 8), "per")])
def test_green_apply(precision, grid, kind):
    bcs = absorbing_z(grid[2]) if kind == "absz" else periodic()
    ocfg, solver, plan, pot = _plan_with_oracle_potential(grid, bcs, precision)
    x = random_field(ocfg.padded_size + (3,), 1)
    y = plan.green_apply(x)
    ref = O.green_conv(x, ocfg, pot.k_square)
    assert rel(y, ref) < OP_TOL[precision]


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_operator_and_preconditioner(precision):
    grid = (32, 32, 16)
    ocfg, solver, plan, pot = _plan_with_oracle_potential(grid, absorbing_z(16), precision)
    x = random_field(ocfg.padded_size + (3,), 2)
    y0 = random_field(ocfg.padded_size + (3,), 3)
    a, b = 0.7 - 0.2j, 1.5 + 0.5j
    y = plan.apply_operator(x, y0, alpha=a, beta=b)
    ref = O.cbs_operator(x, pot.V, ocfg, pot.k_square, alpha=a, beta=b, y=y0)
    assert rel(y, ref) < OP_TOL[precision]
    p = plan.apply_preconditioner(x)
    assert rel(p, O.cbs_preconditioner(x, pot.V, pot.eps_imag)) < OP_TOL[precision]


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_curl(precision):
    grid = (32, 16, 16)
    ocfg, solver, plan, pot = _plan_with_oracle_potential(grid, absorbing_z(16), precision)
    E = random_field(ocfg.padded_size + (3,), 4)
    H = plan.curl_field(E)
    assert rel(H, O.magnetic_field(E, RES, WL)) < OP_TOL[precision]


@pytest.mark.parametrize("precision", ["float64", "float32-math64"])
def test_solve_gmres_96_grid(precision):
    """96-point x/y axes (radix 3) through the whole solve: the 96x96x64 serving grid shape at a smaller z."""
    ref, out, solver = _solve_pair((96, 96, 8), 6.0, precision)
    assert rel(out.E, ref.E) < SOLVE_TOL[precision]
    assert rel(out.H, ref.H) < SOLVE_TOL[precision]


def test_batched_operator_equals_single():
    grid = (32, 32, 16)
    ocfg, solver, plan, pot = _plan_with_oracle_potential(grid, absorbing_z(16), "float64")
    xs = [random_field(ocfg.padded_size + (3,), s) for s in (5, 6, 7)]
    X = np.stack(xs, axis=-1)
    Y = plan.apply_operator(np.asfortranarray(X))
    for i, x in enumerate(xs):
        y1 = plan.apply_operator(x)
        assert np.array_equal(Y[..., i], y1)


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_build_potential_matches_host_setup(precision):
    grid = (32, 32, 16)
    ocfg, solver = configs(grid, absorbing_z(16), precision=precision)
    eps = bead(grid, 6.0)
    pot = O.build_potential(ocfg, eps, EPS_BG, WL)
    plan = solver.plan()
    info = plan.build_potential(eps, EPS_BG, WL, solver.attenuation_filters(), -1)
    assert info.bornmax == pot.Bornmax
    assert abs(info.eps_imag - pot.eps_imag) <= 1e-12 * pot.eps_imag
    assert abs(info.k_bg - pot.k_bg) <= 1e-12 * pot.k_bg
    x = random_field(ocfg.padded_size + (3,), 8)
    assert rel(plan.apply_operator(x), O.cbs_operator(x, pot.V, ocfg, pot.k_square)) < OP_TOL[precision]


def _solve_pair(grid, radius, precision, method="gmres", tol=1e-6, bcs=None, sources=None):
    bcs = bcs or absorbing_z(grid[2])
    ls = {"gmres": F.KrylovJL_GMRES(ortho="mgs"), "bicgstab": F.KrylovJL_BICGSTAB(),
          "richardson": F.BornSeries()}[method]
    ocfg, solver = configs(grid, bcs, tol=tol, precision=precision, linear_solver=ls, method=method)
    eps = bead(grid, radius)
    osrc, fsrc = sources if sources is not None else xpol()
    ref = O.solve(ocfg, osrc, eps, EPS_BG)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, fsrc, F.Medium(eps, EPS_BG))
    return ref, out, solver


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
def test_solve_gmres(precision):
    ref, out, solver = _solve_pair((32, 32, 16), 4.0, precision)
    assert out.E.shape == (32, 32, 16, 3)
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
    assert rel(out.E, ref.E) < SOLVE_TOL[precision]
    assert rel(out.H, ref.H) < SOLVE_TOL[precision]


@pytest.mark.parametrize("method,iters", [("bicgstab", 20), ("richardson", 40), ("gmres", 30)])
def test_fixed_iteration_seam_fp64(method, iters):
    """_solve_cbs_scattering seam (fm_solve_source) with a fixed iteration budget (tolerance 0):
    the k-th iterate of each method must match the oracle's k-th iterate."""
    grid = (16, 16, 8)
    ocfg, solver = configs(grid, absorbing_z(8), precision="float64")
    eps = bead(grid, 3.0)
    pot = O.build_potential(ocfg, eps, EPS_BG, WL)
    Ei, Hi = O.incident_field(xpol()[0], ocfg, EPS_BG)
    S = pot.V[..., None] * Ei + (1j * pot.eps_imag) * Ei
    b = O.green_conv(S, ocfg, pot.k_square)
    A = lambda v: O.cbs_operator(v, pot.V, ocfg, pot.k_square)
    M = lambda v: O.cbs_preconditioner(v, pot.V, pot.eps_imag)
    fn = {"bicgstab": O.bicgstab, "richardson": O.richardson, "gmres": O.gmres}[method]
    ref = fn(A, M, b, b.copy(), 0.0, 0.0, iters)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    opts = F._lib.fm_solve_opts()
    opts.method = {"gmres": 0, "bicgstab": 1, "richardson": 2}[method]
    opts.ortho = F._lib.FM_ORTHO_MGS
    opts.maxiters = iters
    opts.reltol = 0.0
    opts.abstol = 0.0
    E, H, info, st = plan.solve_source(S, opts)
    assert st == F._lib.FM_NOT_CONVERGED
    assert info[0].iterations == ref.iters == iters
    assert rel(E, ref.x) < 1e-10
    assert rel(H, O.magnetic_field(ref.x, RES, WL)) < 1e-10


def test_solve_periodic_and_coherent_sources():
    k = np.array([0.0, 0.3, np.sqrt(1 - 0.09)])
    o_src = [O.PlaneWave(WL, [1, 0, 0], k), O.PlaneWave(WL, [1, 0, 0], [0, -0.3, np.sqrt(1 - 0.09)])]
    f_src = [F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=k),
             F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, -0.3, np.sqrt(1 - 0.09)])]
    ref, out, solver = _solve_pair((16, 16, 16), 3.0, "float64", bcs=periodic(), sources=(o_src, f_src))
    assert rel(out.E, ref.E) < 1e-10
    assert rel(out.H, ref.H) < 1e-10


def test_solve_batch_equals_single_fp64():
    grid = (16, 16, 8)
    ocfg, solver = configs(grid, absorbing_z(8), precision="float64", linear_solver=F.KrylovJL_GMRES(ortho="mgs"))
    eps = bead(grid, 3.0)
    med = F.Medium(eps, EPS_BG)
    srcs = [F.PlaneWaveSource(wavelength=WL, polarization=[1, 0, 0], k_vector=[0, 0, 1]),
            F.PlaneWaveSource(wavelength=WL, polarization=[0, 1, 0], k_vector=[0, 0, 1]),
            F.PlaneWaveSource(wavelength=WL, polarization=[0, 1, 0], k_vector=[0.6, 0, 0.8])]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        outs = F.solve_batch(solver, srcs, med)
        for s, o in zip(srcs, outs):
            one = F.solve(solver, s, med)
            assert rel(o.E, one.E) < 1e-12
            assert rel(o.H, one.H) < 1e-12


def test_invalid_inputs_raise():
    grid = (16, 16, 8)
    ocfg, solver = configs(grid, absorbing_z(8))
    with pytest.raises(ValueError):
        F.solve(solver, xpol()[1], F.Medium(np.ones((8, 8, 8), complex), EPS_BG))
    bad = np.ones(grid, complex) * EPS_BG
    bad[3, 3, 3] = np.nan
    with pytest.raises(F._lib.FMError):
        F.solve(solver, xpol()[1], F.Medium(bad, EPS_BG))
    with pytest.raises(F._lib.FMError):
        # axis lengths above 256 that are not powers of two have no transform in this build
        F.ConvergentBornSolver(resolution=RES, grid_size=(300, 16, 8), boundary_conditions=F.PeriodicBoundaryCondition()).plan()


@pytest.mark.parametrize("precision,restart", [("float64", 20), ("float32-math64", 0), ("float32-math64", 20)])
def test_solve_gmres_split_z_average(precision, restart):
    """Absorbing z padded to 512 (the large configuration's z axis): the two shifted z branches run as two z
    passes.  GMRES(20) as the large configuration runs it, and full GMRES.  FP64 follows the oracle to the
    iteration.  The FP32-storage form's distance to FP64 grows with the length of the domain on this 8x8 bead
    (padded z 128 / 256 / 512: 4e-7 / 4e-6 / 2e-4 after 100 / 100 / 124 iterations, with MGS as with CGS), so
    here it is held to 5e-4 and to the oracle's residual estimate within 2 %."""
    grid = (8, 8, 256)
    bcs = absorbing_z(grid[2])
    ls = F.KrylovJL_GMRES(ortho="mgs" if precision == "float64" else "cgs", gmres_restart=restart)
    ocfg, solver = configs(grid, bcs, tol=1e-6, precision=precision, linear_solver=ls, method="gmres")
    assert solver.padded_size()[2] == 512
    eps = bead(grid, 3.0)
    osrc, fsrc = xpol()
    ref = O.solve(ocfg, osrc, eps, EPS_BG, restart=restart)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        out = F.solve(solver, fsrc, F.Medium(eps, EPS_BG))
    if precision == "float64":
        assert solver.iteration_count == ref.iterations
    if precision == "float64":
        assert rel(out.E, ref.E) < SOLVE_TOL[precision]
        assert rel(out.H, ref.H) < SOLVE_TOL[precision]
    else:
        assert rel(out.E, ref.E) < 5e-4 and rel(out.H, ref.H) < 5e-4
        assert abs(solver.residual_history[-1] - ref.residual) < 0.02 * ref.residual
