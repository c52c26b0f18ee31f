"""Generate the golden fixtures in this directory from the CPU oracle.

The reference (Julia) cannot run in this environment, so these vectors pin the
oracle's own output: tests check that the oracle still reproduces them and that
libfmcuda matches them.  Regenerate with:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import cbs_oracle as O  # noqa: E402

RES = (50e-9,) * 3
EPS_BG = 1.33 ** 2
WL = 500e-9


def case_solve():
    g = (16, 16, 8)
    bz = O.AbsorbingBC(g[2] * RES[2], g[2] * RES[2], 1.0)
    cfg = O.SolverConfig(RES, g, (O.PeriodicBC(), O.PeriodicBC(), bz), tolerance=1e-6)
    eps = O.phantom_bead(g, [2.25], 3.0, permittivity_bg=EPS_BG)
    src = O.PlaneWave(WL, [1, 0, 0], [0, 0, 1])
    r = O.solve(cfg, src, eps, EPS_BG)
    np.savez_compressed(os.path.join(HERE, "solve_16x16x8_bead.npz"), eps=eps, E=r.E, H=r.H,
                        iterations=r.iterations, residuals=np.array(r.residuals),
                        eps_imag=r.potential.eps_imag, bornmax=r.potential.Bornmax)


def case_green():
    g = (8, 16, 8)
    bz = O.AbsorbingBC(g[2] * RES[2], g[2] * RES[2], 1.0)
    cfg = O.SolverConfig(RES, g, (O.PeriodicBC(), O.PeriodicBC(), bz))
    eps = O.phantom_bead(g, [2.25], 2.5, permittivity_bg=EPS_BG)
    pot = O.build_potential(cfg, eps, EPS_BG, WL)
    rng = np.random.default_rng(20261203)
    x = rng.standard_normal(cfg.padded_size + (3,)) + 1j * rng.standard_normal(cfg.padded_size + (3,))
    np.savez_compressed(os.path.join(HERE, "green_8x16x8.npz"), eps=eps, V=pot.V, x=x,
                        green=O.green_conv(x, cfg, pot.k_square), op=O.cbs_operator(x, pot.V, cfg, pot.k_square),
                        k_bg=pot.k_bg, eps_imag=pot.eps_imag)


if __name__ == "__main__":
    case_solve()
    case_green()
    print("written")
