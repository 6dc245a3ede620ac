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


class _FakeHam:
    def __init__(self, dimension):
        self.dimension = dimension


class _FakePropagator:
    """Stands in for BatchedPropagator on CPU: the 'yield' of a trajectory is
    its state's first entry, so the gather order can be checked."""

    def __init__(self, dims):
        self.hamiltonians = [_FakeHam(d) for d in dims]

    def propagate(self, states, times, *, system_index, lifetime_us):
        import numpy as np

        class R:
            pass

        r = R()
        r.yields = np.array([float(s[0]) for s in states])
        return r


def _shard_main(rank, world, port, out):
    import numpy as np
    import torch.distributed as dist

    from rpm_b200.distributed import propagate_sharded, rank_shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prop = _FakePropagator([221184, 13824, 864])
        index = np.array([0] * 3 + [1] * 5 + [2] * 8)
        states = [np.array([float(k)]) for k in range(index.size)]
        span = rank_shard([prop.hamiltonians[k].dimension for k in index], dist)
        _, got_span, yields = propagate_sharded(prop, states, index, [0.0, 1.0], dist, lifetime_us=1.0)
        out.put((rank, span, got_span, yields.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_propagate_cost_balanced_shards():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, s0, g0, y0), (_, s1, g1, y1) = results
    assert s0 == g0 and s1 == g1 and s0[0] == 0 and s0[1] == s1[0] and s1[1] == 16
    # the three 221,184-dim trajectories outweigh the other thirteen: rank 0 gets
    # the first two only, rank 1 the rest
    assert s0 == (0, 2)
    assert y0 == y1 == [float(k) for k in range(16)]
