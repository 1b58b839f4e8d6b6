"""Pins the oracle against the reference's own known-answer tests (CPU only).

The reference ships no golden files; its tests hold these KATs for the build path:
  src/dag_builder.zig:420-521   morton, empty, single voxel, dense == points == fn, dedup
  src/rt_prims.zig:140-160      exact prims and AABBs of a 3-voxel DAG
  tests/cpu_test.zig:758-1060   GPU algorithm (CpuExec) vs CPU builder, edits vs rebuild,
                                LOD vs largest key per coarse cell, chunk batch == single
  tests/cpu_test.zig:296-406    dense vs points node words, out-of-range -> InvalidArgument
Each test below restates one of them against the oracle. The reference's PRNG
(Zig DefaultPrng) is not reproducible here, so seeded inputs of our own replace it.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from pyrit_b200 import workloads as wl


def _lookup_dense(d, dense, log2):
    n = 1 << log2
    idx = np.arange(n ** 3, dtype=np.uint64)
    pts = np.stack([idx % n, (idx // n) % n, idx // (n * n)], axis=1).astype(np.uint32)
    got = orc.lookup_many(log2, d.nodes, d.leaves, d.attrs, d.root, pts)
    return got


def test_morton_kat():  # dag_builder.zig:420-426
    assert orc.morton(1, 0, 0) == 1
    assert orc.morton(0, 1, 0) == 2
    assert orc.morton(0, 0, 1) == 4
    # round trip incl. the 21-bit extreme
    for v in [(0, 0, 0), (1, 0, 0), (0, 1, 0), (5, 9, 1023), (0x1FFFFF, 3, 0x12345)]:
        m = orc.morton(*v)
        dec = tuple(sum(((m >> (3 * i + a)) & 1) << i for i in range(21)) for a in range(3))
        assert dec == v


def test_empty_geometry():  # dag_builder.zig:428-433
    d = orc.cpu_build_points(3, np.zeros((0, 4), np.uint32))
    assert d.nodes[d.root] & 0xFF == 0
    assert orc.lookup_many(3, d.nodes, d.leaves, d.attrs, d.root, np.array([[1, 2, 3]], np.uint32))[0] == 0


def test_single_voxel():  # dag_builder.zig:435-442
    d = orc.cpu_build_points(4, np.array([[5, 6, 7, 42]], np.uint32))
    assert d.voxel_count == 1
    got = orc.lookup_many(4, d.nodes, d.leaves, d.attrs, d.root, np.array([[5, 6, 7], [5, 6, 6]], np.uint32))
    assert list(got) == [42, 0]


def _sphere_noise(log2, seed):
    n = 1 << log2
    rng = np.random.default_rng(seed)
    idx = np.arange(n ** 3)
    x, y, z = idx % n, (idx // n) % n, idx // (n * n)
    c = (n - 1) / 2
    inside = ((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2 < (0.375 * n) ** 2) | (rng.integers(0, 50, n ** 3) == 0)
    vals = (1 + rng.integers(0, 1000, n ** 3)).astype(np.uint32)
    return np.where(inside, vals, 0).astype(np.uint32)


@pytest.mark.parametrize("seed", [1234, 7])
def test_dense_points_fn_equal(seed):  # dag_builder.zig:444-498
    log2 = 5
    dense = _sphere_noise(log2, seed)
    pts = wl.dense_to_points(dense, log2)
    np.random.default_rng(seed).shuffle(pts)  # order must not matter
    a = orc.cpu_build_dense(log2, dense)
    b = orc.cpu_build_points(log2, pts)
    c = orc.cpu_build_fn_dense(log2, dense)
    assert np.array_equal(a.nodes, b.nodes)
    assert np.array_equal(a.leaves, b.leaves)
    assert np.array_equal(a.attrs, b.attrs)
    assert np.array_equal(a.nodes, c.nodes) and a.root == c.root
    assert np.array_equal(_lookup_dense(a, dense, log2), dense)
    assert a.voxel_count == len(pts)


def test_dedup_period8():  # dag_builder.zig:500-521
    log2 = 6
    n = 1 << log2
    idx = np.arange(n ** 3)
    x, y, z = idx % n, (idx // n) % n, idx // (n * n)
    dense = (((x % 8) + (y % 8)) < ((z % 8) + 2)).astype(np.uint32)
    d = orc.cpu_build_dense(log2, dense, store_attrs=False)
    assert len(d.nodes) <= 4 * 10
    got = orc.lookup_many(log2, d.nodes, d.leaves, None, d.root,
                          np.stack([x, y, z], 1).astype(np.uint32))
    assert np.array_equal(got, dense)


def test_points_out_of_range_invalid():  # cpu_test.zig:296-406 (out of range -> INVALID_ARGUMENT)
    with pytest.raises(ValueError):
        orc.cpu_build_points(3, np.array([[8, 0, 0, 1]], np.uint32))
    with pytest.raises(ValueError):
        orc.cpu_build_points(3, np.array([[0, 0, 0, 0]], np.uint32))
    with pytest.raises(ValueError):
        orc.cpu_build_points(2, np.zeros((0, 4), np.uint32))


def test_rt_prims_kat():  # rt_prims.zig:140-160
    pts = np.array([[1, 2, 3, 7], [30, 31, 17, 8], [31, 31, 17, 9]], np.uint32)
    d = orc.cpu_build_points(5, pts)
    prims, aabbs = orc.rt_prims_extract(d, 4)
    assert len(prims) // 16 == 2
    rec = prims.reshape(-1, 16)
    cell = rec[:, 8:16].copy().view(np.uint64).ravel()
    attr_base = rec[:, 4:8].copy().view(np.uint32).ravel()
    a = aabbs.reshape(-1, 6)
    assert abs(a[0, 0] - 1) < 0.01 and abs(a[0, 5] - 4) < 0.01
    assert attr_base[0] == 0
    assert cell[1] == 1 | (1 << 21) | (1 << 42)
    assert attr_base[1] == 1
    assert abs(a[1, 0] - 30) < 0.01 and abs(a[1, 3] - 32) < 0.01


def _scene_points(log2, seed=21, dups=200):
    """cpu_test.zig:758-784: scene as a shuffled point list with duplicates and outliers."""
    dense = wl.scene_dense(log2)
    pts = wl.dense_to_points(dense, log2)
    np.random.default_rng(seed).shuffle(pts)
    d = pts[:dups].copy()
    pts = np.concatenate([pts, d, np.array([[0xFFFFFFFF, 0, 0, 5], [1 << log2, 0, 0, 5]], np.uint32)])
    return dense, pts


def test_gbuild_vs_cpu_builder_with_prims():  # cpu_test.zig:758-807
    log2 = 6
    dense, pts = _scene_points(log2)
    g = orc.gb_build(log2, 4, pts)
    ref = orc.cpu_build_fn_dense(log2, dense)
    assert np.array_equal(_lookup_dense(g, dense, log2) if False else
                          orc.lookup_many(log2, g.nodes, g.leaves, g.attrs, g.root,
                                          _all_points(log2)), _lookup_dense(ref, dense, log2))
    assert g.voxel_count == ref.voxel_count
    assert np.array_equal(g.attrs, ref.attrs)
    assert np.array_equal(g.leaves, ref.leaves)
    prims, aabbs = orc.rt_prims_extract(ref, 4)
    assert g.prim_count == len(prims) // 16
    gr = g.prims.reshape(-1, 16)
    rr = prims.reshape(-1, 16)
    assert np.array_equal(gr[:, 4:16], rr[:, 4:16])  # attr_base and cell
    assert np.array_equal(g.aabbs.view(np.uint32), aabbs.view(np.uint32))
    # P2: canonical node buffers equal, and the GPU layout is already canonical
    cn, croot, shared, lu = orc.canonicalize(log2, ref.nodes, ref.root)
    gn, groot, gshared, glu = orc.canonicalize(log2, g.nodes, g.root)
    assert gshared == 0
    assert np.array_equal(gn, g.nodes) and groot == g.root
    if shared == 0:
        assert np.array_equal(cn, gn) and croot == groot


def _all_points(log2):
    n = 1 << log2
    idx = np.arange(n ** 3, dtype=np.uint64)
    return np.stack([idx % n, (idx // n) % n, idx // (n * n)], axis=1).astype(np.uint32)


def test_gbuild_edits_equal_rebuild():  # cpu_test.zig:809-850
    base = np.array([[x, 0, z, 0x10] for z in range(32) for x in range(32)], np.uint32)
    b1 = orc.gb_build(5, 3, base)
    edits = [[10, y, 10, 0x20] for y in range(1, 20)] + [[x, 0, 3, 0] for x in range(8)] + [[20, 0, 20, 0x30]]
    b2 = orc.gb_build(5, 3, np.array(edits, np.uint32), b1.keys, b1.attrs)
    final = []
    for v in base:
        if v[2] == 3 and v[0] < 8:
            continue
        a = 0x30 if (v[0] == 20 and v[2] == 20) else v[3]
        final.append([v[0], v[1], v[2], a])
    final += [[10, y, 10, 0x20] for y in range(1, 20)]
    ref = orc.cpu_build_points(5, np.array(final, np.uint32))
    pts = _all_points(5)
    assert np.array_equal(orc.lookup_many(5, b2.nodes, b2.leaves, b2.attrs, b2.root, pts),
                          orc.lookup_many(5, ref.nodes, ref.leaves, ref.attrs, ref.root, pts))
    assert b2.voxel_count == len(final)
    # empty geometry
    b3 = orc.gb_build(4, 4, np.zeros((0, 4), np.uint32))
    assert b3.node_words == 2 and b3.root == 0 and b3.prim_count == 0
    assert orc.lookup_many(4, b3.nodes, b3.leaves, b3.attrs, b3.root, np.array([[1, 1, 1]], np.uint32))[0] == 0


def test_gbuild_downsample_largest_key():  # cpu_test.zig:964-999
    log2 = 6
    dense = wl.scene_dense(log2)
    pts = wl.dense_to_points(dense, log2)
    full = orc.gb_build(log2, 3, pts)
    for shift in (1, 2, 3):
        lod = orc.gb_downsample(log2, 3, full.keys, full.attrs, shift)
        best = {}
        for x, y, z, a in pts.tolist():
            c = (x >> shift, y >> shift, z >> shift)
            k = orc.local_key(x, y, z)
            if c not in best or k > best[c][0]:
                best[c] = (k, a)
        ref_pts = np.array([[c[0], c[1], c[2], v[1]] for c, v in best.items()], np.uint32)
        ref = orc.cpu_build_points(log2 - shift, ref_pts)
        allp = _all_points(log2 - shift)
        assert np.array_equal(orc.lookup_many(log2 - shift, lod.nodes, lod.leaves, lod.attrs, lod.root, allp),
                              orc.lookup_many(log2 - shift, ref.nodes, ref.leaves, ref.attrs, ref.root, allp))


def _shell_chunks(k=5, cap=8000, n=32):
    """cpu_test.zig:1001-1030: chunk c holds a spherical shell; chunk 3 stays empty."""
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
        m = len(sel)
        attrs = np.array([wl.lib().wl_attr_of(int(x[i] + c), int(y[i]), int(z[i])) for i in sel], np.uint32)
        vox[c * cap:c * cap + m] = np.stack([x[sel], y[sel], z[sel], attrs], 1)
        cnt[c] = m
    offs = np.concatenate([[0], np.cumsum(cnt)]).astype(np.uint32)
    return vox, cnt, offs


def test_gbuild_chunks_equal_single():  # cpu_test.zig:1001-1060
    k, cap, log2 = 5, 8000, 5
    vox, cnt, offs = _shell_chunks(k, cap)
    b = orc.gb_build_chunks(log2, 4, cap, vox, offs)
    assert b.roots[3] == 0xFFFFFFFF
    pts = _all_points(log2)
    allprims = b.prims.reshape(-1, 16)
    for c in range(k):
        if c == 3:
            continue
        s = orc.gb_build(log2, 4, vox[c * cap:c * cap + cnt[c]])
        count_c = int(b.nodes[b.roots[c] + 1])
        assert count_c == s.voxel_count
        got = orc.lookup_many(log2, b.nodes, b.leaves, b.attrs[b.first_voxel[c]:], b.roots[c], pts)
        exp = orc.lookup_many(log2, s.nodes, s.leaves, s.attrs, s.root, pts)
        assert np.array_equal(got, exp)
        sp = s.prims.reshape(-1, 16)
        gp = allprims[b.first_prim[c]:b.first_prim[c] + len(sp)]
        assert np.array_equal(sp[:, 4:16], gp[:, 4:16])


def test_canonicalizer_reports_cross_level_sharing():
    # a level-3 node [1, 64, 0] whose ref 0 is the level-2 node [1, 64, 0] itself
    nodes = np.array([1, 64, 0, 1, 64, 0], np.uint32)
    # root at offset 3 (level 3 for log2 4): child 0 -> node 0 (level 2) -> leaf 0
    cn, root, shared, _ = orc.canonicalize(4, nodes, 3)
    assert shared == 0 and root == 3 and list(cn) == [1, 64, 0, 1, 64, 0]
    cn, root, shared, _ = orc.canonicalize(4, nodes, 0)   # node 0 reached as level 3 and as level 2
    assert shared == 1 and list(cn) == [1, 64, 0, 1, 64, 0] and root == 3


def test_worldedit_overlay_equals_last_wins():
    """worldedit.zig apply/compact/append == stable 'append edits, last wins' when each
    chunk's edit list names every coordinate at most once (what prepareEdits builds)."""
    rng = np.random.default_rng(3)
    k, cap, log2 = 4, 6000, 5
    vox, cnt, offs = _shell_chunks(k, cap)
    edits, eoff = [], [0]
    for c in range(k):
        pos = rng.choice(32 ** 3, 300, replace=False)
        for p in pos:
            a = 0 if rng.integers(2) else int(rng.integers(1, 9))
            edits.append([p % 32, (p // 32) % 32, p // 1024, a])
        eoff.append(len(edits))
    edits = np.array(edits, np.uint32)
    eoff = np.array(eoff, np.uint32)
    ov, oc = orc.we_apply_all(k, cap * 2, np.concatenate([vox.reshape(k, cap, 4),
                                                          np.zeros((k, cap, 4), np.uint32)], 1).reshape(-1, 4),
                              cnt, edits, eoff)
    ov = ov.reshape(k, cap * 2, 4)
    for c in range(k):
        merged = {}
        for v in vox[c * cap:c * cap + cnt[c]].tolist():
            merged[tuple(v[:3])] = v[3]
        for e in edits[eoff[c]:eoff[c + 1]].tolist():
            merged[tuple(e[:3])] = e[3]
        want = sorted((p, a) for p, a in merged.items() if a != 0)
        got = sorted((tuple(v[:3]), v[3]) for v in ov[c, :oc[c]].tolist())
        assert got == want


def test_pyrd_header():
    d = orc.cpu_build_points(4, np.array([[5, 6, 7, 42]], np.uint32))
    b = orc.pyrd_bytes(4, d.root, d.voxel_count, d.nodes, d.leaves, d.attrs)
    assert b[:4] == b"PYRD"
    h = np.frombuffer(b[4:20], np.uint32)
    assert list(h) == [1, 4, d.root, 1]
    assert len(b) == 52 + 4 * len(d.nodes) + 8 * len(d.leaves) + 4 * 1
