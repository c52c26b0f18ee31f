"""fm_green_apply_noalloc: the Green application that allocates no device memory.

Some callers cannot let a library call cudaMalloc: they own every device buffer through their own
pooled allocator, or run under a fixed device-memory budget.  They pass device buffers they own and
the library works in one static device array.  The test checks the new entry point, called through
the C ABI on device buffers, against the existing fm_green_apply (plan, host buffers) on two calls in a
row, with the tolerances of the other operator tests.  The file is named to run last.
"""
import ctypes

import numpy as np
import pytest

from _cases import EPS_BG, WL, absorbing_z, bead, configs, random_field, rel
from oracle import cbs_oracle as O

import fmcuda as F
from fmcuda import _lib

pytestmark = pytest.mark.gpu

TOL = {"float64": 1e-12, "float32": 2e-6, "float32-math64": 2e-7}


def _to_device(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a.astype(dtype).ravel(order="F"))).cuda()


@pytest.mark.parametrize("precision", ["float64", "float32", "float32-math64"])
def test_noalloc_matches_green_apply(precision):
    torch = pytest.importorskip("torch")
    grid = (32, 32, 16)
    ocfg, solver = configs(grid, absorbing_z(grid[2]), precision=precision)
    pot = O.build_potential(ocfg, bead(grid, 4.0), EPS_BG, WL)
    plan = solver.plan()
    plan.set_potential(pot.V, pot.k_bg, pot.eps_imag, WL)
    shp = ocfg.padded_size + (3, 2)
    xs = [random_field(shp, 11), random_field(shp, 12)]
    refs = [plan.green_apply(x) for x in xs]
    dt = np.complex128 if precision == "float64" else np.complex64
    xd = [_to_device(torch, x, dt) for x in xs]
    yd = torch.empty_like(xd[0])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    lib = _lib.lib()
    free0 = None
    for x_dev, ref in zip(xd, refs):
        torch.cuda.synchronize()
        st = lib.fm_green_apply_noalloc(ctypes.byref(plan.desc), pot.k_bg, pot.eps_imag, 2,
                                        ctypes.c_void_p(x_dev.data_ptr()), ctypes.c_void_p(yd.data_ptr()), stream)
        assert st == _lib.FM_OK, lib.fm_last_error().decode()
        free = torch.cuda.mem_get_info()[0]
        if free0 is not None:
            assert free == free0  # the second call allocated nothing
        free0 = free
        y = yd.cpu().numpy().reshape(shp, order="F")
        assert rel(y, ref) < TOL[precision]
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
