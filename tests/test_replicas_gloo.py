"""Replicas over right-hand sides on two gloo ranks (CPU): sharding, the maximum of per-rank timings, and the
gather of per-rank fields to rank 0 in the original order.  Each rank solves its share with the CPU oracle as the
stand-in for the GPU solve (which the GPU tests cover); the control flow is the one the multi-GPU bench and solve
path use."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fmcuda import replicas as R


def test_shard_round_robin_and_by_cost():
    assert [R.shard(7, 3, r) for r in range(3)] == [[0, 3, 6], [1, 4], [2, 5]]
    costs = [5.0, 1.0, 1.0, 1.0, 4.0, 1.0]
    parts = [R.shard(6, 2, r, costs) for r in range(2)]
    assert sorted(parts[0] + parts[1]) == list(range(6))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= 1.0
    with pytest.raises(ValueError):
        R.shard(3, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


RES = (50e-9,) * 3
WL = 500e-9
EPS_BG = 1.33 ** 2
GRID = (8, 8, 4)


def _oracle_case():
    from oracle import cbs_oracle as O
    t = GRID[2] * RES[2]
    cfg = O.SolverConfig(RES, GRID, (O.PeriodicBC(), O.PeriodicBC(), O.AbsorbingBC(t, t, 1.0)))
    eps = O.phantom_bead(GRID, [2.25], 2.0, permittivity_bg=EPS_BG)
    srcs = [O.PlaneWave(WL, [1, 0, 0], [0, 0, 1]), O.PlaneWave(WL, [0, 1, 0], [0, 0, 1]),
            O.PlaneWave(WL, [0, 1, 0], [0.6, 0, 0.8]), O.PlaneWave(WL, [1, 0, 0], [0, 0.6, 0.8]),
            O.PlaneWave(WL, [0, 0, 1], [0.6, 0.8, 0])]
    return cfg, eps, srcs


def _oracle_solve_batch(cfg, sources, eps):
    from oracle import cbs_oracle as O
    from fmcuda.fields import ElectromagneticField
    out = []
    for s in sources:
        r = O.solve(cfg, s, eps, EPS_BG)
        out.append(ElectromagneticField(r.E, r.H, RES, WL))
    return out


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "frequencymaxwell.jl_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from fmcuda import replicas as R
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = R.max_over_ranks(1.0 + rank)
        cfg, eps, srcs = _oracle_case()
        idx, mine, allf = R.solve_batch_sharded(_oracle_solve_batch, cfg, srcs, eps)
        q.put((rank, t, idx, None if allf is None else [(f.E, f.H) for f in allf]))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        rank, t, idx, allf = q.get(timeout=120)
        res[rank] = (t, idx, allf)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][0] == res[1][0] == 2.0          # max of 1.0 and 2.0 on every rank
    assert res[0][1] == [0, 2, 4] and res[1][1] == [1, 3]
    assert res[1][2] is None
    cfg, eps, srcs = _oracle_case()               # gathered in the original order, bit for bit
    for (E, H), f in zip(res[0][2], _oracle_solve_batch(cfg, srcs, eps)):
        assert np.array_equal(E, f.E) and np.array_equal(H, f.H)
