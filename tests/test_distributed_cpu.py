"""Multi-rank host logic on CPU: two gloo ranks (no GPU)."""

import os
import socket

import pytest

from rpm_b200.distributed import gather_yields, max_over_ranks, shard_bounds, trajectory_costs


def test_shard_bounds_cover_and_balance():
    costs = trajectory_costs([221184] * 10 + [13824] * 20 + [864] * 30)
    for world in (1, 2, 3, 4, 8):
        b = shard_bounds(costs, world)
        assert b[0][0] == 0 and b[-1][1] == costs.size
        assert all(b[k][1] == b[k + 1][0] for k in range(world - 1))
        loads = [costs[s:e].sum() for s, e in b]
        assert max(loads) <= costs.sum() / world + costs.max()
    assert shard_bounds([1.0, 1.0], 4)[-1] == (2, 2)
    with pytest.raises(ValueError):
        shard_bounds([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        counts = [3, 2]
        mine = torch.arange(counts[rank], dtype=torch.float64) + 10 * rank
        allv = gather_yields(mine, dist)
        t = max_over_ranks(1.5 + rank, dist)
        out.put((rank, allv.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_and_max():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, allv, t in results:
        assert allv == [0.0, 1.0, 2.0, 10.0, 11.0]
        assert t == 2.5
