"""fm_green_apply_noalloc: the Green application that allocates no device memory.

Some callers cannot let a library call cudaMalloc: they own every device buffer through their own
pooled allocator, or run under a fixed device-memory budget.  They pass device buffers they own and
the library works in one static device array.  The test calls the new entry point through the C ABI on
device buffers, twice in a row on the same buffers, and checks each result against the existing
fm_green_apply (plan, host buffers) and against the CPU oracle's conv!(G, x), with the tolerances of
the other operator tests.  It covers the averaged absorbing-z branch and the periodic branch, in the three
precisions, with one and two right-hand sides.  The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

from _cases import EPS_BG, WL, absorbing_z, bead, configs, periodic, random_field, rel
from oracle import cbs_oracle as O

from fmcuda import _lib

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-12, "float32": 2e-6, "float32-math64": 2e-7}
CASES = [((32, 32, 16), "absz", 2), ((32, 16, 32), "per", 2), ((16, 32, 8), "absz", 1)]


def _to_device(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a.astype(dtype).ravel(order="F"))).cuda()


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
@pytest.mark.parametrize("grid,kind,nrhs", CASES)
def test_noalloc_matches_green_apply_and_oracle(precision, grid, kind, nrhs):
    torch = pytest.importorskip("torch")
    bcs = absorbing_z(grid[2]) if kind == "absz" else periodic()
    ocfg, solver = configs(grid, bcs, precision=precision)
    pot = O.build_potential(ocfg, bead(grid, min(grid) / 4), EPS_BG, WL)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    shp = ocfg.padded_size + (3, nrhs)
    xs = [random_field(shp, 11), random_field(shp, 12)]
    refs = [plan.green_apply(x) for x in xs]
    oracle = [np.stack([O.green_conv(np.asfortranarray(x[..., b]), ocfg, pot.k_square) for b in range(nrhs)], axis=-1)
              for x in xs]
    dt = np.complex128 if precision == "float64" else np.complex64
    xd = [_to_device(torch, x, dt) for x in xs]
    yd = torch.empty_like(xd[0])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = _lib.lib()
    for i, (x_dev, ref, orc) in enumerate(zip(xd, refs, oracle)):
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = lib.fm_green_apply_noalloc(ctypes.byref(plan.desc), pot.k_bg, pot.eps_imag, nrhs,
                                        ctypes.c_void_p(x_dev.data_ptr()), ctypes.c_void_p(yd.data_ptr()), stream)
        assert st == _lib.FM_OK, lib.fm_last_error().decode()
        if i > 0:
            assert torch.cuda.mem_get_info()[0] == free_before  # a repeated call allocates nothing
        y = yd.cpu().numpy().reshape(shp, order="F")
        assert rel(y, ref) < TOL[precision]
        assert rel(y, orc) < TOL[precision]
    solver.release()


def test_noalloc_rejects_sizes_beyond_the_scratch():
    d = _lib.fm_plan_desc()
    d.grid[:] = [128, 128, 64]
    d.pad[:] = [0, 0, 32]
    d.resolution[:] = [50e-9] * 3
    d.absorbing[:] = [0, 0, 1]
    d.precision = _lib.FM_PREC_F32
    lib = _lib.lib()
    x = ctypes.c_void_p(256)
    y = ctypes.c_void_p(1 << 40)
    st = lib.fm_green_apply_noalloc(ctypes.byref(d), 1.67e7, 7.7e13, 4, x, y, None)
    assert st == _lib.FM_ERR_INVALID
    assert b"scratch" in lib.fm_last_error()
