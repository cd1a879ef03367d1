"""Replica plumbing on two CPU ranks (gloo): request sharding and the
max / sum reductions that bench.py applies to per-rank timings."""
import os
import socket

import pytest

from npme_b200 import multi, serving


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx = multi.max_over_ranks([1.0 + rank, 10.0 - rank], dist)
        sm = multi.sum_over_ranks([rank + 1.0], dist)
        q.put((rank, mx, sm))
    finally:
        dist.destroy_process_group()


def test_shards_are_disjoint_and_complete():
    reqs = serving.serving_stream(count=37, n_max=2000, seed=3)
    world = 3
    parts = [multi.shard_requests(reqs, r, world) for r in range(world)]
    ids = sorted(r.rid for p in parts for r in p)
    assert ids == sorted(r.rid for r in reqs)
    assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_single_rank_reductions_are_identity():
    assert multi.max_over_ranks([2.5, 3]) == [2.5, 3.0]
    assert multi.sum_over_ranks([4]) == [4.0]


def test_two_gloo_ranks_reduce_to_max_and_sum():
    torch_mp = pytest.importorskip("torch.multiprocessing")
    ctx = torch_mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm in out:
        assert mx == [2.0, 10.0]
        assert sm == [3.0]
