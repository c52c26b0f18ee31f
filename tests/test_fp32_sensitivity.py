"""Why the FP32-storage forms lose accuracy on long domains (CPU, oracle only).

On an 8x8x256 grid with an absorbing z boundary (padded z 512) and one bead, GMRES as the reference runs it stops at
its iteration limit (124 iterations, preconditioned residual ~3e-3): the returned iterate is not converged, and it
is sensitive to perturbations of the Krylov process.  Rounding only the stored Krylov basis to complex64 after each
orthogonalisation -- everything else in FP64 -- already moves the iterate by more than 1e-5, and so does rounding
only the preconditioned operator's outputs.  The FP32-storage forms of the library do both, so on such domains
they cannot meet 1e-5 whatever their arithmetic; only FP64 storage can.  The same algorithm in FP64 reproduces
the oracle's iterate to 1e-10.

A defect correction (GMRES restarted every m iterations from the residual recomputed in FP64, the inner basis and
operator outputs in complex64) does remove the storage error: it agrees with the same scheme run in FP64 to about
1e-6.  But a restart changes the method: the restarted iterate, in FP64, is several per cent away from the full-GMRES
iterate at the iteration limit, so no such scheme reproduces the reference's result on a non-converged domain.
"""
import numpy as np
import pytest

from oracle import cbs_oracle as O

pytestmark = pytest.mark.slow

RES = (50e-9,) * 3
WL = 500e-9
EPS_BG = 1.33 ** 2


def _round32(a):
    return a.astype(np.complex64).astype(np.complex128)


def _gmres_rounded(cfg, pot, src, round_basis, round_ops):
    """Full GMRES (CGS, warm start b, left preconditioner) with optional complex64 rounding of the stored basis
    and of the preconditioned operator's outputs; returns the cropped E and H and the iteration count."""
    V, ksq = pot.V, pot.k_square
    Ei, Hi = O.incident_field(src, cfg, EPS_BG)
    S = V[..., None] * Ei + (1j * pot.eps_imag) * Ei
    b = O.green_conv(S, cfg, ksq)
    rop = _round32 if round_ops else (lambda a: a)
    rba = _round32 if round_basis else (lambda a: a)
    b = rop(b)

    def MA(v):
        return rop(O.cbs_preconditioner(O.cbs_operator(v, V, cfg, ksq), V, pot.eps_imag))

    x = b.copy()
    r0 = rop(O.cbs_preconditioner(b - O.cbs_operator(x, V, cfg, ksq), V, pot.eps_imag))
    beta = np.linalg.norm(r0)
    basis = [rba(r0 / beta)]
    itmax = max(2 * pot.Bornmax, 100)
    eps = 1e-8 + 1e-6 * beta
    H = np.zeros((itmax + 1, itmax), complex)
    g = np.zeros(itmax + 1, complex)
    g[0] = beta
    for j in range(itmax):
        w = MA(basis[j])
        h = np.array([np.vdot(v, w) for v in basis])
        w = w - sum(hi * v for hi, v in zip(h, basis))
        hb = np.linalg.norm(w)
        H[:j + 1, j] = h
        H[j + 1, j] = hb
        basis.append(rba(w / hb))
        y = np.linalg.lstsq(H[:j + 2, :j + 1], g[:j + 2], rcond=None)[0]
        if np.linalg.norm(H[:j + 2, :j + 1] @ y - g[:j + 2]) <= eps:
            break
    x = x + sum(yi * v for yi, v in zip(y, basis))
    Hs = O.magnetic_field(x, cfg.resolution, WL)
    return cfg.crop(x + Ei), cfg.crop(Hs + Hi), j + 1


@pytest.fixture(scope="module")
def long_domain():
    grid = (8, 8, 256)
    t = grid[2] * RES[2]
    cfg = O.SolverConfig(RES, grid, (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(t, t, 1.0)))
    eps = O.phantom_bead(grid, [2.25], 3.0, permittivity_bg=EPS_BG)
    src = O.PlaneWave(WL, [1, 0, 0], [0, 0, 1])
    ref = O.solve(cfg, src, eps, EPS_BG)
    assert cfg.padded_size[2] == 512 and ref.iterations == 124 and not ref.solved
    return cfg, src, ref


def test_long_domain_iterate_is_sensitive_to_fp32_storage(long_domain):
    cfg, src, ref = long_domain
    pot = ref.potential
    E, H, it = _gmres_rounded(cfg, pot, src, False, False)
    assert it == ref.iterations
    assert O.rel_l2(E, ref.E) < 1e-9 and O.rel_l2(H, ref.H) < 1e-9
    E, H, _ = _gmres_rounded(cfg, pot, src, True, False)  # basis stored in complex64 only
    assert O.rel_l2(E, ref.E) > 1e-5
    E, H, _ = _gmres_rounded(cfg, pot, src, False, True)  # operator outputs in complex64 only
    assert O.rel_l2(E, ref.E) > 1e-5


def _defect_corrected(cfg, pot, src, m, total, rounded):
    """GMRES restarted every m iterations from the FP64 preconditioned residual M^{-1}(b - A x), x kept in FP64;
    inside a cycle the basis and the operator outputs are rounded to complex64 when `rounded`.  Warm start b,
    `total` operator applications in all; returns the cropped E."""
    V, ksq = pot.V, pot.k_square
    Ei, _ = O.incident_field(src, cfg, EPS_BG)
    b = O.green_conv(V[..., None] * Ei + (1j * pot.eps_imag) * Ei, cfg, ksq)
    rop = _round32 if rounded else (lambda a: a)
    x = b.copy()
    used = 0
    while used < total:
        r = O.cbs_preconditioner(b - O.cbs_operator(x, V, cfg, ksq), V, pot.eps_imag)
        beta = np.linalg.norm(r)
        basis = [rop(r / beta)]
        k = min(m, total - used)
        H = np.zeros((k + 1, k), complex)
        g = np.zeros(k + 1, complex)
        g[0] = beta
        for j in range(k):
            w = rop(O.cbs_preconditioner(O.cbs_operator(basis[j], V, cfg, ksq), V, pot.eps_imag))
            h = np.array([np.vdot(v, w) for v in basis])
            w = w - sum(hi * v for hi, v in zip(h, basis))
            H[:j + 1, j] = h
            H[j + 1, j] = np.linalg.norm(w)
            basis.append(rop(w / H[j + 1, j]))
        y = np.linalg.lstsq(H, g, rcond=None)[0]
        x = x + sum(yi * v for yi, v in zip(y, basis[:k]))
        used += k
    return cfg.crop(x + Ei)


def test_defect_correction_fixes_precision_not_the_iterate(long_domain):
    cfg, src, ref = long_domain
    pot = ref.potential
    E64 = _defect_corrected(cfg, pot, src, 20, ref.iterations, rounded=False)
    E32 = _defect_corrected(cfg, pot, src, 20, ref.iterations, rounded=True)
    assert O.rel_l2(E32, E64) < 1e-5   # measured 1.5e-6: the FP64 defect removes the storage error
    assert O.rel_l2(E64, ref.E) > 1e-2  # measured 0.19: the restarted method lands elsewhere
