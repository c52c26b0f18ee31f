"""CPU check of the block (s-step) GMRES algebra: the numpy restatement in ``_blockgmres`` takes the iterates of
the oracle's full GMRES (Krylov.jl semantics), for every block size, with stops inside a block and tolerance
stops.  The same algebra, on the device, is checked against the oracle in test_gpu_block_gmres.py."""
import numpy as np
import pytest

from _blockgmres import block_gmres, leja
from _cases import EPS_BG, RES, WL, absorbing_z, bead, configs, xpol
from oracle import cbs_oracle as O


def _problem(n=240, seed=3):
    rng = np.random.default_rng(seed)
    K = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(2 * n) * 0.9
    A = np.eye(n) - K @ np.diag(rng.uniform(0.2, 1.0, n))
    d = rng.uniform(0.5, 2.0, n) + 0.3j
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return (lambda v: A @ v), (lambda v: v / d), b


@pytest.mark.parametrize("s", [2, 3, 4, 5, 8])
@pytest.mark.parametrize("itmax", [40, 23])
def test_block_gmres_takes_the_gmres_iterates(s, itmax):
    """No tolerance: every block size runs to the iteration limit, which 23 puts inside a block."""
    A, M, b = _problem()
    ref = O.gmres(A, M, b, b.copy(), 0.0, 0.0, itmax)
    out = block_gmres(A, M, b, b.copy(), 0.0, 0.0, itmax, s)
    assert out.iters == ref.iters == itmax
    assert np.linalg.norm(out.x - ref.x) <= 1e-12 * np.linalg.norm(ref.x)
    assert abs(out.residuals[-1] - ref.residuals[-1]) <= 1e-9 * ref.residuals[-1]


@pytest.mark.parametrize("s", [4, 8])
def test_block_gmres_stops_where_gmres_stops(s):
    A, M, b = _problem(seed=5)
    ref = O.gmres(A, M, b, b.copy(), 0.0, 1e-6, 200)
    out = block_gmres(A, M, b, b.copy(), 0.0, 1e-6, 200, s)
    assert ref.solved and out.solved
    assert out.iters == ref.iters
    assert np.linalg.norm(out.x - ref.x) <= 1e-12 * np.linalg.norm(ref.x)


def test_block_gmres_on_the_cbs_operator():
    """The preconditioned CBS operator of a small bead, 60 non-converged iterations, s = 8."""
    grid = (16, 16, 8)
    ocfg, _ = configs(grid, absorbing_z(8))
    pot = O.build_potential(ocfg, bead(grid, 3.0), EPS_BG, WL)
    osrc, _ = xpol()
    E_inc, _ = O.incident_field(osrc, ocfg, EPS_BG)
    S = pot.V[..., None] * E_inc + (1j * pot.eps_imag) * E_inc
    b = O.green_conv(S, ocfg, pot.k_square)
    A = lambda v: O.cbs_operator(v, pot.V, ocfg, pot.k_square)
    M = lambda v: O.cbs_preconditioner(v, pot.V, pot.eps_imag)
    ref = O.gmres(A, M, b, b.copy(), 0.0, 0.0, 60)
    out = block_gmres(A, M, b, b.copy(), 0.0, 0.0, 60, 8)
    assert out.iters == ref.iters == 60
    assert O.rel_l2(out.x, ref.x) < 1e-10


def test_leja_order():
    pts = [1.0, -1.0, 0.5j, 2.0, -0.25]
    out = leja(pts)
    assert out[0] == 2.0 and sorted(out, key=str) == sorted(pts, key=str)
    # each next point maximises the product of distances to the points before it
    for k in range(1, len(out)):
        prod = lambda z: np.prod([abs(z - w) for w in out[:k]])
        assert all(prod(out[k]) >= prod(z) - 1e-15 for z in out[k:])
