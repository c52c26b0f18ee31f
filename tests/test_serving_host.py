"""Host side of the serving loop (no GPU): slot sizing under the memory budget and the seeded request
stream.  fm_engine_slot_bytes is host arithmetic, so it runs without a device."""
import numpy as np

import fmcuda as F
from fmcuda import serving as SV


def test_slot_plan_fits_budget_and_batches_small_grids():
    for basis in (20, 60, 100):
        plan = SV.slot_plan(SV.SERVING_SHAPES, 150e9, basis, "float32-math64")
        used = 0
        for shape, slots in plan.items():
            sv = F.ConvergentBornSolver(resolution=(50e-9,) * 3, grid_size=shape,
                                        boundary_conditions=SV.serving_boundaries(shape), precision="float32-math64")
            d = F._lib.fm_plan_desc()
            d.grid[:] = list(shape)
            d.pad[:] = list(sv.padding())
            d.precision = F._lib.FM_PREC_F32_MATH64
            per = F._lib.lib().fm_engine_slot_bytes(d, basis)
            n = np.prod(sv.padded_size())
            assert per >= 3 * n * 8 * (basis + 1)
            used += slots * per
            assert slots >= 1
        assert used <= 150e9 or all(v == 1 for v in plan.values())
        assert plan[(64, 64, 32)] > plan[(128, 128, 64)] >= plan[(256, 256, 128)]


def test_serving_boundaries_pad_z_to_twice_the_grid():
    for shape in SV.SERVING_SHAPES:
        sv = F.ConvergentBornSolver(resolution=(50e-9,) * 3, grid_size=shape,
                                    boundary_conditions=SV.serving_boundaries(shape))
        p = sv.padded_size()
        assert p[:2] == shape[:2] and p[2] == 2 * shape[2]


def test_request_stream_is_seeded_and_poisson():
    a = SV.serving_requests(40, rate=200.0, shapes=((32, 32, 16), (64, 32, 32)), max_angles=5, seed=9,
                            beads=3, radius_range=(2, 5))
    b = SV.serving_requests(40, rate=200.0, shapes=((32, 32, 16), (64, 32, 32)), max_angles=5, seed=9,
                            beads=3, radius_range=(2, 5))
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.array_equal(x.medium.permittivity, y.medium.permittivity) for x, y in zip(a, b))
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert 0.05 < arr[-1] < 0.6          # 40 arrivals at a mean 5 ms apart
    assert {r.shape for r in a} == {(32, 32, 16), (64, 32, 32)}
    for r in a:
        assert 1 <= len(r.sources) <= 5
        for s in r.sources:
            assert abs(np.linalg.norm(s.k_vector) - 1) < 1e-12
            assert abs(np.vdot(s.polarization, s.k_vector)) < 1e-12


def test_block_engine_slot_bytes_include_block_vectors():
    grid, basis = (32, 32, 16), 112
    d = F._lib.fm_plan_desc()
    d.grid[:] = list(grid)
    d.pad[:] = [0, 0, grid[2] // 2]
    d.precision = F._lib.FM_PREC_F32_MATH64
    n = grid[0] * grid[1] * 2 * grid[2]
    L = F._lib.lib()
    cgs = L.fm_engine_slot_bytes_ortho(d, basis, F._lib.FM_ORTHO_CGS)
    blk = L.fm_engine_slot_bytes_ortho(d, basis, F._lib.FM_ORTHO_BLOCK)
    assert cgs == L.fm_engine_slot_bytes(d, basis)
    assert blk - cgs >= 3 * n * 16 * 9  # 9 FP64 block vectors
    plan = SV.slot_plan(SV.SERVING_SHAPES, 150e9, basis, "float32-math64", ortho="block")
    assert all(v >= 1 for v in plan.values())
