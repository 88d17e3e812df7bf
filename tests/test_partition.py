"""Sharding one fixed ensemble over ranks (hawassi_c_b200/partition.py) on CPU:
the LPT split of the members by expected device time, and the one end-of-run
gather of per-member scalars over two gloo ranks (the GPU job uses the same code
over NCCL, one process per GPU, with no collective while the members step)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hawassi_c_b200 import decks, partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ensemble_costs(n=256):
    out = []
    for s in range(n):
        pm = decks.ensemble_member_params(s)
        out.append(partition.member_cost(pm["nx"], pm["length"], pm["depth"], 100.0))
    return out


@pytest.mark.parametrize("n_ranks", [1, 2, 3, 4, 8])
def test_partition_covers_and_balances(n_ranks):
    costs = _ensemble_costs()
    shards = partition.greedy_partition(costs, n_ranks)
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(costs)))                 # every member exactly once
    loads = partition.shard_loads(costs, shards)
    lower = max(max(costs), sum(costs) / n_ranks)          # no split can beat this
    assert max(loads) <= 4.0 / 3.0 * lower                 # the LPT guarantee
    assert max(loads) <= 1.02 * lower                      # and in practice within 2 %
    assert shards == partition.greedy_partition(list(costs), n_ranks)   # deterministic


def test_partition_cost_model():
    # a 16384-point member costs more than a 2048-point one of the same depth and span
    a = partition.member_cost(2048, 102.4, 1.0, 100.0)
    b = partition.member_cost(16384, 819.2, 1.0, 100.0)
    assert b / a == pytest.approx(8 * 14 / 11, rel=1e-3)   # same dx up to the (Nx - 1) spacing
    # deeper water: faster fastest mode, more steps
    assert partition.expected_steps(4096, 204.8, 2.0, 1.0) > partition.expected_steps(4096, 204.8, 0.5, 1.0)
    with pytest.raises(ValueError):
        partition.greedy_partition([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_row(m):
    return [100.0, 1000 + 7 * m, 100 + m, m % 5, 0, 1e-3 * (m + 1)]


def _worker(rank, world, port, n, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from hawassi_c_b200 import partition as pt
        costs = [float(10 + (m * 37) % 17) for m in range(n)]
        shards = pt.greedy_partition(costs, world)
        mine = shards[rank]
        tab = pt.gather_member_scalars(mine, [_fake_row(m) for m in mine], n, "cpu")
        q.put((rank, mine, tab))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_and_gather():
    world, n = 2, 37
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, mine, tab = q.get(timeout=120)
        res[r] = (mine, tab)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0][0] + res[1][0]) == list(range(n)) and not set(res[0][0]) & set(res[1][0])
    want = np.array([_fake_row(m) for m in range(n)])
    for r in range(world):
        assert res[r][1].shape == (n, len(partition.SCALARS))
        assert np.array_equal(res[r][1], want)
