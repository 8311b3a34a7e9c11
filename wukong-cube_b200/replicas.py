"""Replica mode on more than one GPU.

Queries are independent and the whole store fits one GPU, so N GPUs run N replicas: one
process per GPU, each holding the full store and answering its own contiguous share of the
query stream.  There is no collective on the data path; the only collective is the reduction of
each rank's device time to the maximum over ranks (whole-job time), and a gather of per-rank
counts where a caller wants them.  (The reference's multi-server mode partitions vertices and
ships rows between servers per step, sparql.hpp:741-808; on one node that exchange buys
nothing while every GPU can hold the whole graph.)
"""
import torch
import torch.distributed as dist


def shard(n_items, rank, world):
    """Contiguous [lo, hi) share of n_items for `rank`; shares differ by at most one item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(value, device="cpu"):
    """The maximum of a per-rank float over all ranks (the rank's own value without a group)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device="cpu"):
    """The sum of a per-rank integer over all ranks."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())
