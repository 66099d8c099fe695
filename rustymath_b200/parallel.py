"""Several GPUs, one process each: independent systems are split into contiguous buckets,
one bucket per rank, with no exchange on the data path; results come back by a gather.

rustymath spreads a stack over threads (parallel::stack, core/src/parallel.rs:118-192); here
the same split runs over ranks of a torch.distributed group (NCCL between GPUs; any backend
for the host-side logic). A single large system is not split: each rank solves its own
(replicas), and timings are reduced as the maximum over ranks."""
import torch.distributed as dist

__all__ = ["shard_range", "max_over_ranks", "map_sharded"]


def shard_range(count, rank, world):
    """[lo, hi): rank's contiguous bucket of `count` items, sizes differing by at most one."""
    base, extra = divmod(count, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(seconds, group=None):
    """The largest of every rank's `seconds` (the job's time is the slowest rank's)."""
    import torch
    if not dist.is_available() or not dist.is_initialized():
        return float(seconds)
    backend = dist.get_backend(group)
    dev = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def map_sharded(fn, items, group=None):
    """fn over this rank's bucket of `items` (a list), then every rank's results gathered back
    into the original order on every rank. fn takes and returns a list."""
    if not dist.is_available() or not dist.is_initialized():
        return list(fn(list(items)))
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    lo, hi = shard_range(len(items), rank, world)
    mine = list(fn(list(items[lo:hi])))
    if len(mine) != hi - lo:
        raise ValueError("fn must return one result per item")
    parts = [None] * world
    dist.all_gather_object(parts, (lo, mine), group=group)
    out = [None] * len(items)
    for start, res in parts:
        out[start:start + len(res)] = res
    return out
