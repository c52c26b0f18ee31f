"""Replicas over right-hand sides on two gloo ranks (CPU): sharding, the maximum of per-rank timings, and the
gather of per-rank results to rank 0 in the original order.  The solve function is a stand-in (the GPU solve is
covered by the GPU tests); the control flow is the one the multi-GPU bench and solve path use."""
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


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = R.max_over_ranks(1.0 + rank)

        def fake_solve_batch(solver, sources, medium):
            return [np.full(3, float(s)) * medium for s in sources]

        idx, mine, allf = R.solve_batch_sharded(fake_solve_batch, None, list(range(5)), 10.0)
        q.put((rank, t, idx, None if allf is None else [a.tolist() for a in allf]))
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
    assert res[0][2] == [[10.0 * s] * 3 for s in range(5)]  # gathered in the original order
