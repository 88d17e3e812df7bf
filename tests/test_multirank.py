"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (the GPU runs use the
same code over NCCL, one process per GPU)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, root, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        mx, sm = bench.reduce_ranks([10.0 * (rank + 1), -float(rank)], [float(rank + 1), 0.5], "cpu")
        decks = bench.make_decks(root, rank, 2)
        q.put((rank, mx, sm, [os.path.basename(d) for d in decks]))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_and_deck_sharding(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = {r[0]: r[1:] for r in res}
    for r in range(world):
        mx, sm, names = res[r]
        assert mx == [20.0, 0.0]          # max over ranks of every time-like value
        assert sm == [3.0, 1.0]           # sum over ranks of every count
    # weak scaling: every rank owns its own members (seeds offset by rank)
    assert res[0][2] == ["m00000", "m00001"] and res[1][2] == ["m00002", "m00003"]
