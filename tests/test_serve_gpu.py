"""Served builds: every request's result is the same alone and in the mix of a batch
(bit-exact: the chunk's node words and leaves re-serialised from its root, its
attributes and its prims), and LRU eviction under a small memory budget keeps serving."""
import numpy as np
import pytest

from pyrit_b200 import workloads as wl

from gpu_helpers import dev, subdag

pytestmark = pytest.mark.gpu


def _pool(n_chunks=12, log2s=None):
    from pyrit_b200.serve import ChunkPool
    if log2s is None:
        log2s = [5 if i % 3 else 6 for i in range(n_chunks)]
    log2s = np.array(log2s, np.uint32)
    vox, offs = wl.mix_chunks_device(log2s, 40, 0)
    return ChunkPool(vox, offs, log2s), vox, offs


def _requests(pool, n, seed=0, rate=None):
    from pyrit_b200.serve import Request
    rng = np.random.default_rng(seed)
    arr = np.zeros(n) if rate is None else wl.poisson_arrivals(n, rate, seed)
    out = []
    for i in range(n):
        c = int(rng.integers(0, len(pool)))
        m = int(rng.integers(0, 65))
        out.append(Request(i, c, wl.chunk_edits(int(pool.log2s[c]), m, 1000 + i), float(arr[i])))
    return out


@pytest.mark.parametrize("edges", ["small", "full"])
def test_results_same_alone_and_in_the_mix(edges):
    """small: a pool of 32^3 / 64^3 chunks; full: the served configuration's edges up to
    256^3 (every request drawn from 32^3 .. 256^3 chunks), batches of several MB."""
    import torch
    from pyrit_b200 import gpu_build
    from pyrit_b200.serve import ChunkServer
    if edges == "small":
        pool, vox, offs = _pool()
        reqs = _requests(pool, 40)
        max_vox = 400_000
    else:
        pool, vox, offs = _pool(log2s=[8, 5, 7, 6, 5, 7, 6, 5, 8, 6])
        reqs = _requests(pool, 24, seed=9)
        max_vox = 4_000_000   # a 256^3 chunk (~8.8 M voxels) forms a batch alone, smaller ones share
    srv = ChunkServer(pool, budget_bytes=8 << 30, max_batch_voxels=max_vox, max_inflight=2, rt_log2=5)
    stats = srv.serve(reqs, realtime=False)
    assert stats.batches >= 3 and stats.max_batch_requests >= 2
    host_vox = vox.cpu().numpy().view(np.uint32)
    cache = {}
    for r in reqs:
        res, host = srv.download(r.rid) if r.rid not in cache else cache[r.rid]
        L = int(pool.log2s[r.chunk])
        pts = np.concatenate([host_vox[offs[r.chunk]:offs[r.chunk + 1]], r.edits])
        alone = gpu_build.build(L, 5, dev(pts), n_new=len(pts)).download()
        if alone.voxel_count == 0:
            assert res.root == 0xFFFFFFFF
            continue
        gw, gl, groot = subdag(L, host.nodes, host.leaves, res.root)
        aw, al, aroot = subdag(L, alone.nodes, alone.leaves, alone.root)
        assert gw == aw and gl == al and groot == aroot, r.rid
        n = int(host.nodes[res.root + 1])
        assert n == alone.voxel_count
        assert np.array_equal(host.attrs[res.first_voxel:res.first_voxel + n], alone.attrs), r.rid
        gp = host.prims.reshape(-1, 16)[res.first_prim:res.first_prim + alone.prim_count]
        assert np.array_equal(gp[:, 4:16], alone.prims.reshape(-1, 16)[:, 4:16]), r.rid
    srv.release_all()
    torch.cuda.synchronize()


def test_lru_eviction_under_small_budget():
    from pyrit_b200.serve import ChunkServer
    pool, vox, offs = _pool(6)
    reqs = _requests(pool, 30, seed=3)
    budget = 16 << 20   # a few batches' results: older ones must be evicted to admit more
    srv = ChunkServer(pool, budget_bytes=budget, max_batch_voxels=150_000, max_inflight=2, rt_log2=5)
    stats = srv.serve(reqs, realtime=False)
    assert stats.evictions > 0
    assert len(stats.latencies_ms) == len(reqs)
    assert srv.arena.peak <= budget and srv.arena.used <= budget
    srv.release_all()


def test_realtime_poisson_stream():
    from pyrit_b200.serve import ChunkServer
    pool, vox, offs = _pool(8)
    reqs = _requests(pool, 200, seed=5, rate=4000.0)
    srv = ChunkServer(pool, budget_bytes=4 << 30, max_batch_voxels=2_000_000, max_inflight=2, rt_log2=5)
    s = srv.serve(reqs, realtime=True).summary()
    assert s["requests"] == 200 and s["p50_ms"] > 0 and s["p99_ms"] >= s["p50_ms"]
    srv.release_all()
