"""Bit-exact parity of the CUDA build with the oracle (restatement of the reference
GPU algorithm, src/device/gbuild.zig + src/gpu_build.zig) on seeded inputs, and
canonical parity with the CPU builder (src/dag_builder.zig). Calls go through the
C ABI (libpyrit_b200.so) via pyrit_b200.gpu_build."""
import numpy as np
import pytest

from oracle import oracle as orc
from pyrit_b200 import workloads as wl

from gpu_helpers import assert_same_build, dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["sort", "grid", "bucket"])
def gb(request):
    """Every test of this module runs three times: voxels ordered by the radix sort, by
    the cell grid and by the brick buckets (the last two where the edge allows them);
    the output must not depend on the path."""
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from pyrit_b200 import gpu_build, native
    path = {"sort": native.PATH_SORT, "grid": native.PATH_GRID, "bucket": native.PATH_BUCKET}[request.param]
    gpu_build.set_tuning(0, 0, 50, path)
    yield gpu_build
    gpu_build.set_tuning(0, 0, 50, native.PATH_AUTO)


def _scene_points(log2, seed=21, dups=200):
    dense = wl.scene_dense(log2)
    pts = wl.dense_to_points(dense, log2)
    np.random.default_rng(seed).shuffle(pts)
    d = pts[:dups].copy()
    pts = np.concatenate([pts, d, np.array([[0xFFFFFFFF, 0, 0, 5], [1 << log2, 0, 0, 5]], np.uint32)])
    return dense, pts


@pytest.mark.parametrize("log2,rt", [(6, 4), (6, 3), (6, 6), (5, 5), (3, 3), (4, 3)])
def test_scene_matches_oracle(gb, log2, rt):
    """tests/cpu_test.zig:758-807 input: shuffled scene with duplicates and outliers."""
    _, pts = _scene_points(log2)
    g = gb.build(log2, rt, dev(pts)).download()
    o = orc.gb_build(log2, rt, pts)
    assert_same_build(g, o, label=f"scene log2={log2} rt={rt}")


def test_heightfield_matches_oracle_and_cpu_builder(gb):
    """64^3 heightfield (plain single-chunk build): P1 bytes vs oracle, P2 canonical vs CPU builder."""
    pts = wl.heightfield(6, 0)
    g = gb.build(6, 4, dev(pts)).download()
    o = orc.gb_build(6, 4, pts)
    assert_same_build(g, o, label="heightfield")
    c = orc.cpu_build_points(6, pts)
    cn, croot, shared, lu = orc.canonicalize(6, c.nodes, c.root)
    assert np.array_equal(g.leaves, c.leaves)
    assert np.array_equal(g.attrs, c.attrs)
    assert shared == 0
    assert np.array_equal(cn, g.nodes) and croot == g.root


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_heightfield_seeds(gb, seed):
    pts = wl.heightfield(6, seed)
    g = gb.build(6, 4, dev(pts)).download()
    assert_same_build(g, orc.gb_build(6, 4, pts), label=f"heightfield seed {seed}")


def test_empty_and_tiny(gb):
    for pts in [np.zeros((0, 4), np.uint32),
                np.array([[5, 6, 7, 42]], np.uint32),
                np.array([[5, 6, 7, 42], [5, 6, 7, 0]], np.uint32),          # deleted again
                np.array([[-1 & 0xFFFFFFFF, 0, 0, 3], [16, 0, 0, 3]], np.uint32),  # all outside
                np.array([[1, 1, 1, 9], [1, 1, 1, 10], [1, 1, 1, 11]], np.uint32)]:  # last wins
        g = gb.build(4, 4, dev(pts), n_new=len(pts)).download()
        assert_same_build(g, orc.gb_build(4, 4, pts), label=f"tiny {pts.tolist()}")


def test_edit_path_matches_oracle(gb):
    """cpu_test.zig:809-850: edits on top of the sorted voxels of a previous build."""
    base = np.array([[x, 0, z, 0x10] for z in range(32) for x in range(32)], np.uint32)
    b1 = gb.build(5, 3, dev(base))
    edits = np.array([[10, y, 10, 0x20] for y in range(1, 20)] + [[x, 0, 3, 0] for x in range(8)] +
                     [[20, 0, 20, 0x30]], np.uint32)
    b2 = gb.build(5, 3, dev(edits), old_keys=b1.keys, old_vals=b1.attrs, n_old=b1.voxel_count).download()
    o1 = orc.gb_build(5, 3, base)
    o2 = orc.gb_build(5, 3, edits, o1.keys, o1.attrs)
    assert_same_build(b2, o2, label="edit")


def test_downsample_matches_oracle(gb):
    log2 = 6
    pts = wl.dense_to_points(wl.scene_dense(log2), log2)
    full = gb.build(log2, 3, dev(pts))
    ofull = orc.gb_build(log2, 3, pts)
    for shift in (1, 2, 3):
        g = gb.downsample(log2, 3, full.keys, full.attrs, full.voxel_count, shift).download()
        o = orc.gb_downsample(log2, 3, ofull.keys, ofull.attrs, shift)
        assert_same_build(g, o, label=f"downsample {shift}")


def _shell_chunks(k=5, cap=8000, n=32):
    vox = np.zeros((k * cap, 4), np.uint32)
    cnt = np.zeros(k, np.uint32)
    idx = np.arange(n ** 3)
    x, y, z = idx % n, (idx // n) % n, idx // (n * n)
    d2 = (x - 15.5) ** 2 + (y - 15.5) ** 2 + (z - 15.5) ** 2
    for c in range(k):
        if c == 3:
            continue
        r = 6 + 2 * c
        sel = np.nonzero((d2 < r * r) & (d2 > (r - 2) ** 2))[0][:cap]
        attrs = np.array([wl.lib().wl_attr_of(int(x[i] + c), int(y[i]), int(z[i])) for i in sel], np.uint32)
        vox[c * cap:c * cap + len(sel)] = np.stack([x[sel], y[sel], z[sel], attrs], 1)
        cnt[c] = len(sel)
    offs = np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint32)
    return vox, cnt, offs


@pytest.mark.parametrize("rt", [4, 3, 5])
def test_chunks_match_oracle(gb, rt):
    """cpu_test.zig:1001-1060 batch (chunk 3 empty) -- bytes, roots, first voxels, first prims."""
    k, cap, log2 = 5, 8000, 5
    vox, cnt, offs = _shell_chunks(k, cap)
    g = gb.build_chunks(log2, rt, k, cap, dev(vox), dev(offs), int(offs[-1])).download()
    o = orc.gb_build_chunks(log2, rt, cap, vox, offs)
    assert_same_build(g, o, chunks=True, label=f"chunks rt={rt}")


def test_many_small_chunks_match_oracle(gb):
    """Many chunks of mixed occupancy (incl. empty ones): the per-segment sort tiling."""
    rng = np.random.default_rng(5)
    k, cap, log2 = 37, 3000, 4
    vox = np.zeros((k * cap, 4), np.uint32)
    cnt = np.zeros(k, np.uint32)
    for c in range(k):
        m = int(rng.integers(0, cap + 1)) if c % 5 else 0
        v = rng.integers(0, 16, (m, 3)).astype(np.uint32)
        a = rng.integers(0, 6, (m, 1)).astype(np.uint32)  # attribute 0 deletes
        vox[c * cap:c * cap + m] = np.concatenate([v, a], 1)
        cnt[c] = m
    offs = np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint32)
    g = gb.build_chunks(log2, 3, k, cap, dev(vox), dev(offs), int(offs[-1])).download()
    o = orc.gb_build_chunks(log2, 3, cap, vox, offs)
    assert_same_build(g, o, chunks=True, label="many chunks")


def test_noise256_with_edits_matches_oracle(gb):
    """256^3 noise grid + 0.5% edit overlay (the headline plain-build workload)."""
    vox = wl.noise_grid(8, 0)
    ed = wl.noise_edits(8, 0)
    pts = np.concatenate([vox, ed])
    b = gb.build(8, 7, dev(pts))
    st = gb.last_stats()
    g = b.download()
    o = orc.gb_build(8, 7, pts)
    assert_same_build(g, o, label="noise256")
    # the memory the build took is the host-side bound, under the reference's 130 B/voxel
    # (tests/cpu_test.zig:1559-1629)
    scratch, outputs = gb.build_memory(8, len(pts), rt_log2_req=7)
    assert (st.scratch_bytes, st.output_bytes) == (scratch, outputs)
    assert (scratch + outputs) / len(pts) < 130


@pytest.mark.parametrize("radix_bits,tile_keys,lf", [(4, 1024, 50), (8, 2048, 70), (11, 4096, 50), (11, 1024, 90),
                                                     (8, 4096, 25), (9, 4096, 50), (10, 2048, 70), (9, 1024, 50),
                                                     (8, 8192, 50), (9, 8192, 70)])
def test_tuning_variants_are_bit_exact(gb, radix_bits, tile_keys, lf):
    """The autotuner's knobs (digit width, tile, load factor) never change the output."""
    _, pts = _scene_points(6)
    o = orc.gb_build(6, 4, pts)
    old = gb.get_tuning()
    try:
        gb.set_tuning(radix_bits, tile_keys, lf, old.path)
        g = gb.build(6, 4, dev(pts)).download()
    finally:
        gb.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    assert_same_build(g, o, label=f"tuning {radix_bits}/{tile_keys}/{lf}")


@pytest.mark.parametrize("radix_bits", [8, 9])
def test_large_sort_tiles_match_oracle(gb, radix_bits):
    """8192-entry sort tiles (512-thread sort blocks, unique in two parts) over many
    tiles, ragged last tile included."""
    pts = np.concatenate([wl.noise_grid(7, 1), wl.noise_edits(7, 1)])
    o = orc.gb_build(7, 5, pts)
    old = gb.get_tuning()
    try:
        gb.set_tuning(radix_bits, 8192, 50, old.path)
        g = gb.build(7, 5, dev(pts)).download()
    finally:
        gb.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    assert len(pts) % 8192 != 0
    assert_same_build(g, o, label=f"tiles 8192, {radix_bits} bits")


def _dup_runs(last_attr, seed=5):
    """Bricks whose run of equal key >> 6 crosses sort tiles: 9000 copies of voxel
    (0,0,0) (the last copy decides: attr `last_attr`, 0 deletes), then its brick
    neighbours and other bricks, so that the brick's first kept voxel lies two tiles
    after the tile where its run begins; and a second brick of 10000 entries."""
    rng = np.random.default_rng(seed)
    a = np.zeros((9000, 4), np.uint32)
    a[:, 3] = rng.integers(1, 200, 9000)
    a[-1, 3] = last_attr
    nb = np.array([[1, 0, 0, 3], [0, 1, 0, 0], [3, 3, 3, 7]], np.uint32)   # (0,1,0) is deleted
    other = np.concatenate([rng.integers(4, 32, (3000, 3)), rng.integers(0, 6, (3000, 1))], 1).astype(np.uint32)
    dups = np.repeat(np.array([[9, 9, 9, 4], [9, 9, 10, 0]], np.uint32), 5000, axis=0)
    return np.concatenate([a, other, nb, dups])


@pytest.mark.parametrize("last_attr", [5, 0])
@pytest.mark.parametrize("tuning", [(8, 4096), (9, 8192), (8, 1024)])
def test_brick_runs_across_tiles(gb, last_attr, tuning):
    pts = _dup_runs(last_attr)
    o = orc.gb_build(5, 3, pts)
    old = gb.get_tuning()
    try:
        gb.set_tuning(tuning[0], tuning[1], 50, old.path)
        g = gb.build(5, 3, dev(pts)).download()
    finally:
        gb.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    assert_same_build(g, o, label=f"duplicate runs, last attr {last_attr}, tuning {tuning}")


def test_brick_runs_all_deleted(gb):
    """A run of one brick's entries over several tiles with nothing kept: no brick."""
    a = np.zeros((10000, 4), np.uint32)
    a[:, 0] = np.arange(10000) % 4
    a[:, 3] = 0
    pts = np.concatenate([a, np.array([[8, 8, 8, 2], [31, 31, 31, 1]], np.uint32)])
    assert_same_build(gb.build(5, 3, dev(pts)).download(), orc.gb_build(5, 3, pts), label="all deleted")


@pytest.mark.parametrize("tuning", [(8, 4096), (9, 8192), (8, 1024)])
def test_brick_runs_with_interleaved_cells(gb, tuning):
    """The sort orders bricks only, so a brick's run keeps its entries in input order
    with their cells interleaved: 12,800 entries cycling over the 64 cells of one brick
    in shuffled order, attributes 0..3 (0 deletes), so that each cell's last entry lies
    anywhere in a run over several tiles and past their ends; out-of-range entries
    (keys without brick bits) interleaved with brick 0's own voxels; other bricks
    around both."""
    rng = np.random.default_rng(23)
    cyc = np.concatenate([rng.permutation(64) for _ in range(200)])
    brick = np.stack([4 + (cyc & 3), 4 + ((cyc >> 2) & 3), 4 + (cyc >> 4), rng.integers(0, 4, len(cyc))], 1)
    b0 = np.concatenate([rng.integers(0, 4, (300, 3)), rng.integers(0, 4, (300, 1))], 1)
    bad = np.concatenate([rng.integers(32, 40, (150, 1)), rng.integers(0, 4, (150, 2)), rng.integers(0, 4, (150, 1))], 1)
    bad = np.concatenate([bad, np.array([[0xFFFFFFFF, 1, 1, 3]] * 150)])
    mixed = np.concatenate([b0, bad])[rng.permutation(600)]
    other = np.concatenate([rng.integers(8, 32, (2000, 3)), rng.integers(0, 4, (2000, 1))], 1)
    pts = np.concatenate([other[:1000], brick, mixed, other[1000:], brick[:100]]).astype(np.uint32)
    o = orc.gb_build(5, 3, pts)
    old = gb.get_tuning()
    try:
        gb.set_tuning(tuning[0], tuning[1], 50, old.path)
        g = gb.build(5, 3, dev(pts)).download()
    finally:
        gb.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    assert_same_build(g, o, label=f"interleaved cells, tuning {tuning}")


@pytest.mark.parametrize("lf", [50, 25])
def test_leaf_table_regions_with_repeated_masks(gb, lf):
    """A leaf table larger than one region (64 MB; here at load factor 25 %) is filled
    region by region (bricks grouped by the region of their mask's home slot, each
    region cleared right before its inserts): 1.5 M bricks of one voxel each at one of
    four places, so four masks repeat ~375 k times each across regions and warps."""
    rng = np.random.default_rng(17)
    cells = rng.choice(128 ** 3, 1_500_000, replace=False)
    bx, by, bz = cells % 128, (cells // 128) % 128, cells // (128 * 128)
    corner = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [3, 3, 3]])[rng.integers(0, 4, len(cells))]
    pts = np.stack([bx * 4 + corner[:, 0], by * 4 + corner[:, 1], bz * 4 + corner[:, 2],
                    rng.integers(1, 6, len(cells))], 1).astype(np.uint32)
    o = orc.gb_build(9, 5, pts)
    old = gb.get_tuning()
    try:
        gb.set_tuning(8, 4096, lf, old.path)
        g = gb.build(9, 5, dev(pts)).download()
    finally:
        gb.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    assert len(o.leaves) == 4
    assert_same_build(g, o, label=f"leaf regions, load factor {lf}")


def test_invalid_arguments(gb):
    from pyrit_b200.native import PyrbError
    pts = dev(np.array([[1, 1, 1, 1]], np.uint32))
    for log2 in (2, 21):
        with pytest.raises(PyrbError) as ei:
            gb.build(log2, 3, pts, n_new=1)
        assert ei.value.code == -1
    with pytest.raises(PyrbError) as ei:
        gb.downsample(6, 3, 0, 0, 0, 4)
    assert ei.value.code == -1


@pytest.mark.parametrize("log2,rt,n", [(11, 7, 60000), (12, 9, 40000), (16, 12, 20000), (20, 3, 3000), (20, 20, 500)])
def test_large_edges_64bit_keys_match_oracle(gb, log2, rt, n):
    """Edges 2^11 .. 2^20 need 64-bit sort keys (3*log2 + 1 > 32 bits): sparse clustered
    points plus outliers and duplicates, bit-exact with the oracle."""
    rng = np.random.default_rng(log2)
    side = 1 << log2
    centers = rng.integers(0, side, (8, 3))
    pts = (centers[rng.integers(0, 8, n)] + rng.integers(-20, 21, (n, 3))) % side
    attrs = rng.integers(0, 5, (n, 1))
    v = np.concatenate([pts, attrs], 1).astype(np.uint32)
    v = np.concatenate([v, v[:50], np.array([[side, 0, 0, 1], [0xFFFFFFFF, 1, 1, 1], [side - 1, side - 1, side - 1, 7]],
                                            np.uint32)])
    g = gb.build(log2, rt, dev(v)).download()
    o = orc.gb_build(log2, rt, v)
    assert_same_build(g, o, label=f"log2={log2}")


@pytest.mark.parametrize("log2,rt,n,passes", [(10, 7, 30000, 6), (20, 3, 3000, 7)])
def test_most_sort_passes_match_oracle(gb, log2, rt, n, passes):
    """The most sort passes a build takes: the sort orders the brick bits (3 log2 - 6),
    so 6 passes for 4-bit digits at edge 2^10 (24 bits) and 7 for 64-bit keys at edge
    2^20 (54 bits), which always take 8-bit digits; each pass has its own dynamic tile
    counter, none shared with the unique, leaf or level kernels."""
    rng = np.random.default_rng(100 + log2)
    side = 1 << log2
    centers = rng.integers(0, side, (4, 3))
    pts = (centers[rng.integers(0, 4, n)] + rng.integers(-12, 13, (n, 3))) % side
    v = np.concatenate([pts, rng.integers(0, 4, (n, 1))], 1).astype(np.uint32)
    v = np.concatenate([v, v[:40]])
    from pyrit_b200 import native
    old = gb.get_tuning()
    try:
        gb.set_tuning(4, 1024, 50, native.PATH_SORT)
        g = gb.build(log2, rt, dev(v)).download()
        assert gb.last_stats().sort_passes == passes
    finally:
        gb.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    assert_same_build(g, orc.gb_build(log2, rt, v), label=f"4-bit digits, log2={log2}")


@pytest.mark.parametrize("seed", [0, 1])
def test_world_edit_overlay_matches_worldedit_then_build_chunks(gb, seed):
    """World path: generated chunk voxels with each chunk's overlay edits merged by the
    build (sort-merge, last entry wins) == the reference's worldedit apply/compact/append
    (src/device/worldedit.zig:26-90) followed by buildChunks, byte for byte. Edit lists
    name every coordinate at most once per chunk, as World.prepareEdits produces them."""
    rng = np.random.default_rng(seed)
    K, log2, cap = 6, 5, 12000
    n = 1 << log2
    vox = np.zeros((K * cap, 4), np.uint32)
    counts = np.zeros(K, np.uint32)
    edits, eoff = [], [0]
    for c in range(K):
        g = wl.mix_chunk(100 + c, log2, seed) if c != 2 else np.zeros((0, 4), np.uint32)
        g = g[:cap // 2]
        vox[c * cap:c * cap + len(g)] = g
        counts[c] = len(g)
        m = int(rng.integers(0, 400))
        pos = rng.choice(n ** 3, m, replace=False)
        for p in pos:
            a = 0 if rng.integers(2) else int(rng.integers(1, 9))
            edits.append([p % n, (p // n) % n, p // (n * n), a])
        eoff.append(len(edits))
    edits = np.array(edits, np.uint32).reshape(-1, 4)
    eoff = np.array(eoff, np.uint32)
    g = gb.build_chunks_edits(log2, 4, K, cap, dev(vox), dev(counts), dev(edits), dev(eoff), int(eoff[-1])).download()
    ov, oc = orc.we_apply_all(K, cap, vox, counts, edits, eoff)
    offs = np.concatenate([[0], np.cumsum(oc)]).astype(np.uint32)
    packed = np.zeros_like(ov)
    for c in range(K):  # buildChunks reads segment c from voxels[c * cap], filled to oc[c]
        packed[c * cap:c * cap + oc[c]] = ov[c * cap:c * cap + oc[c]]
    o = orc.gb_build_chunks(log2, 4, cap, packed, offs)
    assert_same_build(g, o, chunks=True, label="world overlay")


@pytest.mark.parametrize("seed", [0, 1])
def test_world_edit_overlay_with_repeated_coordinates(gb, seed):
    """Edit lists that name a coordinate several times and edits on generated voxels:
    every chunk builds as if its edits were applied after its generated voxels in list
    order (the last entry of a coordinate wins, attribute 0 removes) -- the build of
    the concatenated lists, byte for byte."""
    rng = np.random.default_rng(50 + seed)
    K, log2, cap = 5, 5, 9000
    n = 1 << log2
    vox = np.zeros((K * cap, 4), np.uint32)
    counts = np.zeros(K, np.uint32)
    segs, edits, eoff = [], [], [0]
    for c in range(K):
        g = wl.mix_chunk(500 + c, log2, seed)[:cap // 2] if c != 3 else np.zeros((0, 4), np.uint32)
        vox[c * cap:c * cap + len(g)] = g
        counts[c] = len(g)
        m = int(rng.integers(50, 600))
        e = np.empty((m, 4), np.uint32)
        e[:, :3] = rng.integers(0, n // 2, (m, 3))          # a small corner: many repeats
        if len(g):
            k = min(m // 3, len(g))
            e[:k, :3] = g[rng.integers(0, len(g), k), :3]    # edits on generated voxels
        e[:, 3] = np.where(rng.random(m) < 0.4, 0, rng.integers(1, 9, m))
        edits.append(e)
        eoff.append(eoff[-1] + m)
        segs.append(np.concatenate([g, e]))
    ed = np.concatenate(edits)
    eoff = np.array(eoff, np.uint32)
    got = gb.build_chunks_edits(log2, 4, K, cap, dev(vox), dev(counts), dev(ed), dev(eoff), int(eoff[-1])).download()
    cap2 = max(len(sg) for sg in segs)
    packed = np.zeros((K * cap2, 4), np.uint32)
    for c in range(K):
        packed[c * cap2:c * cap2 + len(segs[c])] = segs[c]
    offs = np.concatenate([[0], np.cumsum([len(sg) for sg in segs])]).astype(np.uint32)
    o = orc.gb_build_chunks(log2, 4, cap2, packed, offs)
    assert_same_build(got, o, chunks=True, label="repeated edits")
