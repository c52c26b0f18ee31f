"""Self-consistency of the oracle: FFT Green apply vs a direct DFT, Krylov solves vs a dense solve,
and the three iterative forms agreeing at convergence."""
import math

import numpy as np

from oracle import cbs_oracle as O


def _direct_green(src, cfg, ksq, shifts):
    """_apply_single_convolution! evaluated with explicit DFT matrices (no FFT)."""
    n = src.shape[:3]
    fr = [2 * math.pi / (n[d] * cfg.resolution[d]) for d in range(3)]
    x = src * O.phase_ramp(n, shifts, False)[..., None]
    F = [np.exp(-2j * np.pi * np.outer(np.arange(m), np.arange(m)) / m) for m in n]
    X = np.einsum("ia,jb,kc,abcd->ijkd", F[0], F[1], F[2], x)
    X = O.green_multiply(X, fr, shifts, ksq)
    Fi = [np.conj(f) / f.shape[0] for f in F]
    y = np.einsum("ia,jb,kc,abcd->ijkd", Fi[0], Fi[1], Fi[2], X)
    return y * O.phase_ramp(n, shifts, True)[..., None]


def _small_case(grid=(8, 8, 4), absorbing=True):
    res = (50e-9,) * 3
    bz = O.AbsorbingBC(grid[2] * res[2], grid[2] * res[2], 1.0) if absorbing else O.PeriodicBC()
    cfg = O.SolverConfig(res, grid, (O.PeriodicBC(), O.PeriodicBC(), bz))
    eps = O.phantom_bead(grid, [2.25], 2.0, permittivity_bg=1.33 ** 2)
    pot = O.build_potential(cfg, eps, 1.33 ** 2, 500e-9)
    return cfg, eps, pot


def test_green_fft_matches_direct_dft():
    cfg, eps, pot = _small_case((6, 8, 4))
    rng = np.random.default_rng(0)
    x = rng.standard_normal(cfg.padded_size + (3,)) + 1j * rng.standard_normal(cfg.padded_size + (3,))
    ref = (_direct_green(x, cfg, pot.k_square, cfg.shifts) +
           _direct_green(x, cfg, pot.k_square, tuple(-s for s in cfg.shifts))) / 2
    assert O.rel_l2(O.green_conv(x, cfg, pot.k_square), ref) < 1e-12


def test_green_fft_matches_direct_dft_absorbing_all_axes():
    """Shifts of 1/4 on x, y and z (absorbing on every axis): both branches against explicit DFT matrices."""
    res = (50e-9,) * 3
    grid = (4, 6, 4)
    bcs = tuple(O.AbsorbingBC(grid[d] * res[d], grid[d] * res[d], 1.0) for d in range(3))
    cfg = O.SolverConfig(res, grid, bcs)
    assert cfg.shifts == (0.25, 0.25, 0.25)
    eps = O.phantom_bead(grid, [2.25], 1.5, permittivity_bg=1.33 ** 2)
    pot = O.build_potential(cfg, eps, 1.33 ** 2, 500e-9)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(cfg.padded_size + (3,)) + 1j * rng.standard_normal(cfg.padded_size + (3,))
    ref = (_direct_green(x, cfg, pot.k_square, cfg.shifts) +
           _direct_green(x, cfg, pot.k_square, tuple(-s for s in cfg.shifts))) / 2
    assert O.rel_l2(O.green_conv(x, cfg, pot.k_square), ref) < 1e-12


def test_krylov_matches_dense_solve():
    cfg, eps, pot = _small_case((4, 4, 2))
    n = int(np.prod(cfg.padded_size)) * 3
    shp = cfg.padded_size + (3,)
    A = lambda v: O.cbs_operator(v, pot.V, cfg, pot.k_square)
    M = lambda v: O.cbs_preconditioner(v, pot.V, pot.eps_imag)
    cols = []
    for i in range(n):
        e = np.zeros(n, complex)
        e[i] = 1
        cols.append(M(A(e.reshape(shp, order="F"))).ravel(order="F"))
    MA = np.stack(cols, axis=1)
    rng = np.random.default_rng(1)
    b = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp))
    xd = np.linalg.solve(MA, M(b).ravel(order="F")).reshape(shp, order="F")
    g = O.gmres(A, M, b, b.copy(), 0.0, 1e-13, n + 5)
    assert O.rel_l2(g.x, xd) < 1e-9
    g20 = O.gmres(A, M, b, b.copy(), 0.0, 1e-13, 2000, restart=20)
    assert O.rel_l2(g20.x, xd) < 1e-8


def test_methods_agree_when_converged():
    cfg, eps, pot = _small_case((8, 8, 4), absorbing=False)
    src = O.PlaneWave(500e-9, [1, 0, 0], [0, 0, 1])
    r = {m: O.solve(cfg, src, eps, 1.33 ** 2, method=m, rtol=1e-12, atol=0.0, itmax=3000)
         for m in ("gmres", "bicgstab")}
    assert r["gmres"].solved
    assert O.rel_l2(r["bicgstab"].E, r["gmres"].E) < 1e-8


def test_green_and_curl_index_differ_for_odd_sizes():
    # dyadic_green.jl:203-208 vs curl.jl:84-86
    assert list(O.green_k_index(5)) == [0, 1, 2, -2, -1]
    assert list(O.curl_k_index(5)) == [0, 1, -3, -2, -1]
    assert list(O.green_k_index(4)) == list(O.curl_k_index(4)) == [0, 1, -2, -1]


def test_bornmax_and_eps_imag_config1():
    # convergent_born.jl:641, 653-660 on the 64x64x32 single-bead configuration
    res = (50e-9,) * 3
    g = (64, 64, 32)
    bz = O.AbsorbingBC(32 * 50e-9, 32 * 50e-9, 1.0)
    cfg = O.SolverConfig(res, g, (O.PeriodicBC(), O.PeriodicBC(), bz))
    eps = O.phantom_bead(g, [2.25], 8.0, permittivity_bg=1.33 ** 2)
    pot = O.build_potential(cfg, eps, 1.33 ** 2, 500e-9)
    assert cfg.padded_size == (64, 64, 64)
    assert pot.Bornmax == 16
    assert pot.eps_imag == __import__("pytest").approx(7.673e13, rel=1e-3)
