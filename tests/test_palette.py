"""Chunk attribute palettes (src/device/palette.zig): the oracle against hand-worked
cases of the reference's rules (CPU), and the CUDA scan/pack against the oracle byte
for byte on random chunks with colliding home slots and on a built chunk batch (GPU)."""
import numpy as np
import pytest

from oracle import oracle as orc

OVER = 0xFFFFFFFF


def _hash(v):
    h = (v * 0x9E3779B1) & 0xFFFFFFFF
    return h ^ (h >> 15)


def test_oracle_palette_rules():
    attrs = np.array([5, 5, 7] + list(range(1, 18)) + [9], np.uint32)
    first = np.array([0, 3, 20, 21, 21], np.uint32)   # last chunk empty
    pal, cnt = orc.palette_scan(attrs, first)
    assert list(cnt) == [2, OVER, 1, 0]
    order = sorted([5, 7], key=lambda v: _hash(v) & 63)
    assert list(pal[0]) == order + [order[0]] * 14          # slot order, padded with the first
    assert list(pal[2]) == [9] * 16 and list(pal[3]) == [0] * 16
    dst, total = orc.palette_layout(first, cnt)
    assert list(dst) == [0, 17, 34, 51] and total == 67
    pool = orc.palette_pack(attrs, first, pal, cnt, dst, total)
    idx = [order.index(v) for v in (5, 5, 7)]
    assert pool[16] == idx[0] | (idx[1] << 4) | (idx[2] << 8)
    assert list(pool[17:34]) == list(range(1, 18))            # overflow: 32-bit attributes
    assert list(pool[51:67]) == [0] * 16


def test_oracle_palette_empty_marker_and_collisions():
    # 0xFFFFFFFF is the table's empty marker: never inserted, packs as index 0
    pal, cnt = orc.palette_scan(np.array([OVER, 3, OVER], np.uint32), np.array([0, 3], np.uint32))
    assert cnt[0] == 1 and pal[0][0] == 3
    # two values with one home slot: the first inserted keeps it
    home = {}
    a = b = None
    for v in range(1, 100000):
        s = _hash(v) & 63
        if s in home:
            a, b = home[s], v
            break
        home[s] = v
    for seq in ([a, b], [b, a]):
        pal, cnt = orc.palette_scan(np.array(seq, np.uint32), np.array([0, 2], np.uint32))
        assert cnt[0] == 2 and list(pal[0][:2]) == seq


def _random_chunks(rng, count):
    sizes = rng.integers(0, 9000, count)
    sizes[::7] = 0
    first = np.concatenate([[0], np.cumsum(sizes)]).astype(np.uint32)
    attrs = np.empty(int(first[-1]), np.uint32)
    for c in range(count):
        k = int(rng.choice([1, 2, 5, 12, 16, 17, 40]))
        vals = rng.integers(1, 1 << 32, k, dtype=np.uint64).astype(np.uint32)
        if c % 3 == 0:   # values that share home slots
            vals = np.array([v for v in range(1, 5000) if _hash(v) & 63 in (3, 4)][:k], np.uint32)
        attrs[first[c]:first[c + 1]] = rng.choice(vals, int(sizes[c]))
    return attrs, first


def _check_against_oracle(attrs_host, attrs_dev, first):
    import torch
    from pyrit_b200 import gpu_build
    pal, cnt = gpu_build.palette_scan(attrs_dev, first)
    opal, ocnt = orc.palette_scan(attrs_host, first)
    assert np.array_equal(cnt, ocnt)
    keep = ocnt != OVER
    assert np.array_equal(pal.cpu().numpy().view(np.uint32)[keep], opal[keep])
    dst, total = gpu_build.palette_layout(first, cnt)
    odst, ototal = orc.palette_layout(first, ocnt)
    assert np.array_equal(dst, odst) and total == ototal
    pool = torch.zeros(max(total, 1), dtype=torch.int32, device="cuda")
    gpu_build.palette_pack(attrs_dev, first, pal, cnt, dst, pool)
    opool = orc.palette_pack(attrs_host, first, opal, ocnt, odst, ototal)
    assert np.array_equal(pool.cpu().numpy().view(np.uint32)[:total], opool)
    return cnt


@pytest.mark.gpu
def test_palette_random_chunks_match_oracle():
    from gpu_helpers import dev
    rng = np.random.default_rng(3)
    attrs, first = _random_chunks(rng, 300)
    cnt = _check_against_oracle(attrs, dev(attrs), first)
    assert (cnt == OVER).any() and (cnt != OVER).any()


@pytest.mark.gpu
def test_palette_of_a_chunk_batch_matches_oracle():
    """The install step after a batch build: palettes over the batch's attributes,
    chunk by chunk (first_voxel of the non-empty chunks, then voxel_count)."""
    from pyrit_b200 import gpu_build, workloads as wl
    log2s = wl.chunk_mix(64, 0)
    vox, offs = wl.mix_chunks_device(log2s, 0, 0)
    b = gpu_build.build_batch(log2s, 5, vox, offs)
    h = b.download()
    nonempty = [c for c in range(len(log2s)) if b.roots[c] != 0xFFFFFFFF]
    first = np.array([b.first_voxel[c] for c in nonempty] + [h.voxel_count], np.uint32)
    _check_against_oracle(h.attrs, b.attrs, first)
    b.free()
