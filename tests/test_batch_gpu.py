"""Batched build of chunks with mixed edges (pyrb_build_batch): every chunk, read from
the shared buffers through its root, equals its own single build (oracle restatement
of the reference GPU algorithm) -- node words and leaves after re-serialising from the
root, attributes, keys and prims."""
import numpy as np
import pytest

from oracle import oracle as orc
from pyrit_b200 import workloads as wl

from gpu_helpers import subdag

pytestmark = pytest.mark.gpu


def _chunk(rng, log2, kind):
    n = 1 << log2
    if kind == "empty":
        return np.zeros((0, 4), np.uint32)
    if kind == "full":
        idx = np.arange(n ** 3)
        return np.stack([idx % n, (idx // n) % n, idx // (n * n), np.full(n ** 3, 3)], 1).astype(np.uint32)
    m = int(rng.integers(1, 3 * n * n))
    pts = rng.integers(0, n, (m, 3)).astype(np.uint32)
    a = rng.integers(0, 6, (m, 1)).astype(np.uint32)          # attribute 0 deletes
    return np.concatenate([pts, a], 1)


def _check(log2s, chunks, edits, rt):
    from pyrit_b200 import gpu_build
    K = len(log2s)
    vo = np.concatenate([[0], np.cumsum([len(c) for c in chunks])]).astype(np.uint32)
    vox = np.concatenate(chunks) if vo[-1] else np.zeros((1, 4), np.uint32)
    eo = None
    ed = None
    if edits is not None:
        eo = np.concatenate([[0], np.cumsum([len(e) for e in edits])]).astype(np.uint32)
        ed = np.concatenate(edits) if eo[-1] else np.zeros((1, 4), np.uint32)
    b = gpu_build.build_batch(np.array(log2s, np.uint32), rt, vox, vo, ed, eo)
    g = b.download()
    lmax, lmin = max(log2s), min(log2s)
    rt_eff = min(max(rt, 3), lmin)
    lb = 3 * lmax
    for c in range(K):
        pts = chunks[c] if edits is None else np.concatenate([chunks[c], edits[c]])
        o = orc.gb_build(log2s[c], rt_eff, pts)
        if o.voxel_count == 0:
            assert g.roots[c] == 0xFFFFFFFF and g.first_voxel[c] == 0xFFFFFFFF, c
            continue
        r = int(g.roots[c])
        assert int(g.nodes[r + 1]) == o.voxel_count, c
        gw, gl, groot = subdag(log2s[c], g.nodes, g.leaves, r)
        ow, ol, oroot = subdag(log2s[c], o.nodes, o.leaves, o.root)
        assert gw == ow and gl == ol and groot == oroot, f"chunk {c} (log2 {log2s[c]})"
        f = int(g.first_voxel[c])
        assert np.array_equal(g.attrs[f:f + o.voxel_count], o.attrs), c
        keys = g.keys[f:f + o.voxel_count]
        assert np.all((keys >> np.uint64(lb)) == c) and np.array_equal(keys & np.uint64((1 << lb) - 1), o.keys), c
        p = int(g.first_prim[c])
        gp = g.prims.reshape(-1, 16)[p:p + o.prim_count]
        op = o.prims.reshape(-1, 16)
        assert np.array_equal(gp[:, 4:16], op[:, 4:16]), c        # attr_base and cell
        assert np.array_equal(g.aabbs.reshape(-1, 6)[p:p + o.prim_count].view(np.uint32),
                              o.aabbs.reshape(-1, 6).view(np.uint32)), c


@pytest.mark.parametrize("seed", [0, 1])
def test_mixed_batch_matches_single_builds(seed):
    rng = np.random.default_rng(seed)
    log2s = [3, 4, 5, 3, 5, 4, 4, 5, 3, 5]
    kinds = ["rand", "rand", "rand", "empty", "full", "rand", "full", "rand", "rand", "empty"]
    chunks = [_chunk(rng, l, k) for l, k in zip(log2s, kinds)]
    _check(log2s, chunks, None, rt=3)


def test_mixed_batch_with_edits_and_rt():
    rng = np.random.default_rng(7)
    log2s = [5, 6, 4, 6, 5]
    chunks = [wl.mix_chunk(i, l, 0) if l >= 5 else _chunk(rng, l, "rand") for i, l in enumerate(log2s)]
    edits = [wl.chunk_edits(l, int(rng.integers(0, 65)), 100 + i) for i, l in enumerate(log2s)]
    _check(log2s, chunks, edits, rt=4)


def test_uniform_batch_equals_chunks_api():
    """Same edge for every chunk: the batch form builds what pyrb_build_chunks builds."""
    rng = np.random.default_rng(3)
    log2s = [4] * 12
    chunks = [_chunk(rng, 4, "rand") for _ in log2s]
    _check(log2s, chunks, None, rt=3)


@pytest.mark.parametrize("radix_bits", [8, 9])
def test_mixed_batch_with_large_sort_tiles(radix_bits):
    """8192-entry sort tiles over segments of many sizes: full 32^3 chunks span four
    tiles, small chunks share none, empty ones take none."""
    from pyrit_b200 import gpu_build, native
    rng = np.random.default_rng(11)
    log2s = [5, 3, 5, 4, 5, 3]
    kinds = ["full", "rand", "rand", "empty", "full", "rand"]
    chunks = [_chunk(rng, l, k) for l, k in zip(log2s, kinds)]
    old = gpu_build.get_tuning()
    try:
        gpu_build.set_tuning(radix_bits, 8192, 50, native.PATH_SORT)
        _check(log2s, chunks, None, rt=3)
    finally:
        gpu_build.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)


# The batched configuration's own chunk sizes: 2 chunks of 256^3, 3 of 128^3 and 20 of
# 32^3 / 64^3 from the chunk-mix generator (heightfield tiled per chunk with caves) in
# one batch. Such a batch gives segments of ~1000 sort tiles next to ones of a single
# tile, the root of a small chunk three levels below the batch's top, and unique passes
# split over many tiles; each chunk must still equal its own single build (the
# reference's batch == single property, tests/cpu_test.zig:1001-1060).
CONFIG2_LOG2S = [8, 5, 6, 7, 5, 5, 6, 8, 5, 7, 6, 5, 5, 6, 5, 7, 5, 6, 5, 5, 6, 5, 5, 6, 5]


@pytest.mark.parametrize("path", ["sort", "grid", "bucket"])
@pytest.mark.parametrize("with_edits", [False, True])
def test_config2_mix_at_full_chunk_sizes(with_edits, path):
    from pyrit_b200 import gpu_build, native
    log2s = CONFIG2_LOG2S
    assert log2s.count(8) == 2 and log2s.count(7) == 3 and len(log2s) == 25
    chunks = [wl.mix_chunk(200 + i, l, 0) for i, l in enumerate(log2s)]
    edits = [wl.chunk_edits(l, 64, 300 + i) for i, l in enumerate(log2s)] if with_edits else None
    gpu_build.set_tuning(0, 0, 50, {"sort": native.PATH_SORT, "grid": native.PATH_GRID,
                                    "bucket": native.PATH_BUCKET}[path])
    try:
        _check(log2s, chunks, edits, rt=5)
    finally:
        gpu_build.set_tuning(0, 0, 50, native.PATH_AUTO)
