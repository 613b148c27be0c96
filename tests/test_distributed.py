"""Multi-process host logic of the N-GPU path, on CPU with gloo (world 2 and
3): point sharding, in-order gathering of per-rank results and the
max-over-ranks timing reduction that bench.py uses."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from adaptive_sparse_grid_bench_b200.sharding import shard_range


def test_shard_range_partitions_exactly():
    for total in (0, 1, 7, 1000, 1 << 24):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0
            for (s0, c0), (s1, _) in zip(spans, spans[1:]):
                assert s0 + c0 == s1
            assert sum(c for _, c in spans) == total
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1


def test_shard_range_rejects_bad_input():
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)
    with pytest.raises(ValueError):
        shard_range(10, 0, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, total, q):
    import torch
    import torch.distributed as dist
    from adaptive_sparse_grid_bench_b200.sharding import gather_in_order, max_over_ranks, shard_range
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, count = shard_range(total, rank, world)
        # stand-in for each rank's evaluation of its points: a known function
        local = torch.arange(start, start + count, dtype=torch.float32) * 0.5
        full = gather_in_order(local, total)
        ok_gather = torch.equal(full, torch.arange(total, dtype=torch.float32) * 0.5)
        slowest = max_over_ranks(10.0 + rank)
        q.put((rank, ok_gather, slowest))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,total", [(2, 1001), (3, 17), (2, 0)])
def test_gloo_gather_and_max(world, total):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, total, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, slowest in results:
        assert ok, f"rank {rank} gathered wrong results"
        assert slowest == 10.0 + (world - 1)
