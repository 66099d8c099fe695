"""The multi-rank logic (rustymath_b200.parallel) on CPU: two gloo ranks on 127.0.0.1 split a
batch into contiguous buckets, gather the results in order and reduce timings to the max."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from rustymath_b200.parallel import shard_range


def test_shard_range_covers_everything_once():
    for count in (0, 1, 7, 20000, 20001):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_range(count, r, world)
                assert 0 <= lo <= hi <= count
                seen.extend(range(lo, hi))
            assert seen == list(range(count))
            sizes = [shard_range(count, r, world)[1] - shard_range(count, r, world)[0] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from rustymath_b200.parallel import map_sharded, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = list(range(11))
        res = map_sharded(lambda xs: [(x, x * x, dist.get_rank()) for x in xs], items)
        t = max_over_ranks(0.5 + rank)
        out.put((rank, res, t))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=100) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, res, t in got:
        assert [r[0] for r in res] == list(range(11))
        assert all(r[1] == r[0] * r[0] for r in res)
        owners = [r[2] for r in res]
        assert owners == [0] * 6 + [1] * 5  # contiguous buckets, the first rank takes the extra item
        assert t == 1.5
