"""Replica plumbing for runs on several GPUs of one node.

A single solve does not shard (it would need an FFT all-to-all and halo
exchanges of the direct sum), so N GPUs run N independent solves: one per
rank for the benchmark workload, a share of the requests per rank for the
serving stream.  The only cross-rank step is the reduction of the timings
to their maximum, so the slowest rank sets the whole-job time.
"""


def shard_requests(requests, rank, world):
    """The requests rank `rank` of `world` serves (round robin by id)."""
    return [r for r in requests if r.rid % world == rank]


def max_over_ranks(values, dist=None, device=None):
    """Element-wise maximum of `values` (floats) over the ranks of the
    default process group (`dist` = torch.distributed, None for one rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def sum_over_ranks(values, dist=None, device=None):
    """Element-wise sum of `values` over the ranks of the default group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]
