"""Sharding of chunk builds over ranks: assignments are complete, disjoint, balanced
and identical on every rank (world_size 2 over gloo on CPU), and the host bookkeeping
combines counts by sum and times by max."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pyrit_b200 import shard


def test_chunk_range_covers_all():
    for total in (0, 1, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            got = [shard.chunk_range(total, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            assert max(h - l for l, h in got) - min(h - l for l, h in got) <= 1
    with pytest.raises(ValueError):
        shard.chunk_range(10, 2, 2)


def test_partition_balanced_and_complete():
    rng = np.random.default_rng(0)
    sizes = rng.choice([32 ** 3, 64 ** 3, 128 ** 3, 256 ** 3], p=[.4, .3, .2, .1], size=1024) // 2
    for world in (1, 2, 4, 8):
        parts = shard.partition_chunks(sizes, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(sizes)))
        loads = [int(sizes[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= sizes.max()


def test_route_requests_least_loaded():
    sizes = np.array([100, 1, 1, 1, 50, 50])
    r = shard.route_requests(sizes, 2)
    assert list(r) == [0, 1, 1, 1, 1, 1]
    r = shard.route_requests(sizes, 2, rates=[1.0, 3.0])
    assert r[0] == 0 and all(x == 1 for x in r[1:4])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        sizes = rng.integers(1, 1 << 20, size=300)
        parts = shard.partition_chunks(sizes, world)
        routes = shard.route_requests(sizes, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, (parts[rank].tolist(), routes.tolist(), shard.chunk_range(300, rank, world)))
        mine = {"voxels": float(sizes[parts[rank]].sum()), "chunks": float(len(parts[rank])),
                "build_ms": 10.0 + rank}
        comb = shard.combine(mine)
        q.put((rank, gathered, comb, int(sizes.sum())))
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, g0, c0, total), (_, g1, c1, _) = res
    assert g0 == g1  # both ranks saw the same assignment from every rank
    parts = [g0[r][0] for r in range(2)]
    assert sorted(parts[0] + parts[1]) == list(range(300)) and not set(parts[0]) & set(parts[1])
    assert g0[0][1] == g0[1][1]   # same routing computed on both ranks
    assert g0[0][2] == (0, 150) and g0[1][2] == (150, 300)
    assert c0 == c1
    assert c0["voxels"] == total and c0["chunks"] == 300 and c0["build_ms"] == 11.0
