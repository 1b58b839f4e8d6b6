"""Path edits (src/device/pathedit.zig): voxels of a finished geometry changed without a
rebuild. CPU: the oracle's edited DAG decodes to the edited voxel set, its attributes
and RT prims equal those of a rebuild. GPU: the CUDA path edit equals the oracle byte
for byte on the pools, prims, boxes and job results (plain and palette attributes,
many jobs at once, a job that empties its geometry, a job whose arena overflows)."""
import numpy as np
import pytest

from oracle import oracle as orc
from pyrit_b200 import workloads as wl

EMPTY, OVERFLOW, REBUILD = 0x2, 0x4, 0x1


def _geometry(log2, rt, seed):
    vox = wl.mix_chunk(seed, log2, 0)
    return vox, orc.gb_build(log2, rt, vox)


def _edits(rng, log2, vox, n, remove_frac=0.4):
    """Random sets, inserts and removes (also of existing voxels), some repeated."""
    e = np.empty((n, 4), np.uint32)
    edge = 1 << log2
    for i in range(n):
        if rng.random() < 0.5 and len(vox):
            x, y, z = vox[rng.integers(len(vox))][:3]
        else:
            x, y, z = rng.integers(0, edge, 3)
        a = 0 if rng.random() < remove_frac else int(rng.integers(1, 9))
        e[i] = (x, y, z, a)
    if n > 4:
        e[n - 1] = e[0]
        e[n - 1, 3] = 7
    return e


def _job(g, log2, rt, n_edits, first=0, nodes_base=None, leaves_base=None, attrs_len=None, node_cap=None,
         attr_a=None):
    levels = max(log2 - 2, 0)
    return dict(node_offset=0, leaf_offset=0, root=g.root, log2_size=log2, attr_src=0, attr_count=g.voxel_count,
                attr_a=attr_a if attr_a is not None else len(g.attrs), attr_b=0, attr_cap=g.voxel_count + n_edits,
                palette=0, pal_src=0, pal_dst=0,
                node_arena=nodes_base if nodes_base is not None else len(g.nodes),
                node_cap=node_cap if node_cap is not None else n_edits * (levels * 10 + 4) + 8,
                leaf_arena=leaves_base if leaves_base is not None else len(g.leaves), leaf_cap=n_edits,
                edit_first=first, edit_count=n_edits, rt_log2=rt, prim_count=g.prim_count, aabbs_keep=0)


def _final_voxels(vox, edits):
    order = sorted(range(len(edits)), key=lambda i: (int(edits[i][2]) >> 2, int(edits[i][1]) >> 2,
                                                      int(edits[i][0]) >> 2))   # stable, as the host orders them
    cur = {(int(x), int(y), int(z)): int(a) for x, y, z, a in vox}
    for i in order:
        x, y, z, a = (int(v) for v in edits[i])
        if a:
            cur[(x, y, z)] = a
        else:
            cur.pop((x, y, z), None)
    return cur


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_path_edit_equals_rebuild(seed):
    log2, rt = 5, 4
    rng = np.random.default_rng(seed)
    vox, g = _geometry(log2, rt, seed)
    ed = _edits(rng, log2, vox, 60)
    job = _job(g, log2, rt, len(ed))
    nodes = np.concatenate([g.nodes, np.zeros(job["node_cap"], np.uint32)])
    leaves = np.concatenate([g.leaves, np.zeros(job["leaf_cap"], np.uint64)])
    attrs = np.concatenate([g.attrs, np.zeros(job["attr_cap"], np.uint32)])
    n2, l2, a2, p2, b2, out = orc.path_edit(nodes, leaves, attrs, [job], ed, g.prims, g.aabbs)
    o = out[0]
    final = _final_voxels(vox, ed)
    assert o["out_count"] == len(final)
    assert not (o["out_flags"] & (EMPTY | OVERFLOW))
    edge = 1 << log2
    idx = np.arange(edge ** 3, dtype=np.uint64)
    pts = np.stack([idx % edge, (idx // edge) % edge, idx // (edge * edge)], axis=1).astype(np.uint32)
    got = orc.lookup_many(log2, n2, l2, a2[o["attr_a"]:o["attr_a"] + o["out_count"]], o["out_root"], pts)
    want = np.array([final.get((int(x), int(y), int(z)), 0) for x, y, z in pts], np.uint32)
    assert np.array_equal(got, want)
    # attributes, prims and boxes equal a rebuild of the edited voxels
    fv = np.array([[x, y, z, a] for (x, y, z), a in final.items()], np.uint32)
    r = orc.gb_build(log2, rt, fv)
    assert np.array_equal(a2[o["attr_a"]:o["attr_a"] + o["out_count"]], r.attrs)
    if not (o["out_flags"] & REBUILD) and len(r.prims) // 16 == g.prim_count:
        gp, rp = p2.reshape(-1, 16), r.prims.reshape(-1, 16)
        assert np.array_equal(gp[:, 4:16], rp[:, 4:16])          # attribute rank and cell
        assert np.array_equal(b2.reshape(-1).view(np.uint32), r.aabbs.view(np.uint32))


def test_oracle_path_edit_empties_and_overflows():
    log2, rt = 5, 4
    vox, g = _geometry(log2, rt, 4)
    small = vox[:40]
    g = orc.gb_build(log2, rt, small)
    ed = small.copy()
    ed[:, 3] = 0                                               # remove everything
    job = _job(g, log2, rt, len(ed))
    nodes = np.concatenate([g.nodes, np.zeros(job["node_cap"], np.uint32)])
    leaves = np.concatenate([g.leaves, np.zeros(job["leaf_cap"], np.uint64)])
    attrs = np.concatenate([g.attrs, np.zeros(job["attr_cap"], np.uint32)])
    *_, out = orc.path_edit(nodes, leaves, attrs, [job], ed, g.prims, g.aabbs)
    assert out[0]["out_flags"] & EMPTY
    job = _job(g, log2, rt, 5, node_cap=6)
    *_, out = orc.path_edit(nodes, leaves, attrs, [job], _edits(np.random.default_rng(0), log2, small, 5, 0.0),
                            g.prims, g.aabbs)
    assert out[0]["out_flags"] & OVERFLOW


def _batch_jobs(rng, palette):
    """Jobs over the chunks of a batch built on the GPU: host pools with arenas and
    attribute targets, random edits per chunk, one chunk emptied, one with an arena
    too small. Returns (pools dict, jobs, edits, prim/box host arrays)."""
    from pyrit_b200 import gpu_build
    log2s = np.array([5, 6, 5, 5, 6, 5, 5, 6], np.uint32)
    chunks = [wl.mix_chunk(40 + c, int(l), 0) for c, l in enumerate(log2s)]
    chunks[3] = chunks[3][:30]
    offs = np.concatenate([[0], np.cumsum([len(c) for c in chunks])]).astype(np.uint32)
    b = gpu_build.build_batch(log2s, 4, np.concatenate(chunks), offs)
    h = b.download()
    roots, fv, fp = b.roots.copy(), b.first_voxel.copy(), b.first_prim.copy()
    b.free()
    nz = [c for c in range(len(log2s)) if roots[c] != 0xFFFFFFFF]
    nodes, leaves, attrs = list(h.nodes), list(h.leaves), list(h.attrs)
    prims, aabbs = h.prims.copy(), h.aabbs.copy()
    n_nodes, n_leaves = len(nodes), len(leaves)
    attr_pool = np.array(attrs, np.uint32)
    counts = first = None
    if palette:
        first = np.array([fv[c] for c in nz] + [h.voxel_count], np.uint32)
        pal, counts = orc.palette_scan(attr_pool, first)
        dst, total = orc.palette_layout(first, counts)
        attr_pool = orc.palette_pack(attr_pool, first, pal, counts, dst, total)
    jobs, edits, node_pos, leaf_pos = [], [], n_nodes, n_leaves
    attr_tail = len(attr_pool)
    extra_attrs = []
    for k, c in enumerate(nz):
        lc = int(log2s[c])
        vox_c = chunks[c]
        n_e = 0 if k == 5 else int(rng.integers(5, 60))
        if c == 3:   # the 30-voxel chunk: remove all of it
            e = vox_c.copy()
            e[:, 3] = 0
            n_e = len(e)
        else:
            e = _edits(rng, lc, vox_c, n_e)
        count = int(h.nodes[roots[c] + 1])
        nxt = [fp[d] for d in nz if d > c]
        pc = (nxt[0] if nxt else len(prims) // 16) - fp[c]
        levels = lc - 2
        node_cap = 4 if k == 4 else n_e * (levels * 10 + 4) + 8
        j = dict(node_offset=0, leaf_offset=0, root=int(roots[c]), log2_size=lc, attr_src=int(fv[c]),
                 attr_count=count, attr_b=0, palette=0, pal_src=0, pal_dst=0, node_arena=node_pos, node_cap=node_cap,
                 leaf_arena=leaf_pos, leaf_cap=n_e, edit_first=len(edits), edit_count=n_e, rt_log2=4,
                 prim_count=int(pc), prim_first=int(fp[c]), aabbs_keep=int(k % 2))
        if palette and counts[k] != 0xFFFFFFFF:
            words = 16 + (count + n_e + 7) // 8
            j.update(palette=1, pal_src=int(dst[k]), attr_src=int(dst[k]) + 16, pal_dst=attr_tail,
                     attr_a=attr_tail + 16, attr_cap=(words - 16) * 8)
        else:
            if palette:
                j["attr_src"] = int(dst[k])
            words = count + n_e
            j.update(attr_a=attr_tail, attr_cap=words)
        attr_tail += words
        node_pos += node_cap
        leaf_pos += n_e
        edits.extend(e.tolist())
        jobs.append(j)
    pools = dict(nodes=np.concatenate([np.array(nodes, np.uint32), np.zeros(node_pos - n_nodes, np.uint32)]),
                 leaves=np.concatenate([np.array(leaves, np.uint64), np.zeros(leaf_pos - n_leaves, np.uint64)]),
                 attrs=np.concatenate([attr_pool, np.zeros(attr_tail - len(attr_pool), np.uint32)]))
    return pools, jobs, np.array(edits, np.uint32).reshape(-1, 4), prims, aabbs


@pytest.mark.gpu
@pytest.mark.parametrize("palette", [False, True])
def test_cuda_path_edit_matches_oracle(palette):
    import ctypes
    import torch
    from pyrit_b200 import gpu_build, native
    from gpu_helpers import dev
    rng = np.random.default_rng(7 if palette else 8)
    pools, jobs, edits, prims, aabbs = _batch_jobs(rng, palette)
    n2, l2, a2, p2, b2, want = orc.path_edit(pools["nodes"], pools["leaves"], pools["attrs"], jobs, edits,
                                             prims, aabbs)
    dn, dl, da = dev(pools["nodes"]), dev(pools["leaves"]), dev(pools["attrs"])
    dp = torch.from_numpy(prims.copy()).cuda()
    db = torch.from_numpy(aabbs.copy()).cuda()
    cj = []
    for jd in jobs:
        j = native.PathEditJob()
        for k, v in jd.items():
            if k != "prim_first":
                setattr(j, k, v)
        j.prims = dp.data_ptr() + 16 * jd["prim_first"] if jd["prim_count"] else 0
        j.aabbs = db.data_ptr() + 24 * jd["prim_first"] if jd["prim_count"] else 0
        cj.append(j)
    gpu_build.path_edit(dn, dl, da, cj, edits)
    for w, g in zip(want, cj):
        assert (g.out_root, g.out_count, g.out_flags) == (w["out_root"], w["out_count"], w["out_flags"])
    flags = [w["out_flags"] for w in want]
    assert any(f & EMPTY for f in flags) and any(f & OVERFLOW for f in flags)
    assert np.array_equal(dn.cpu().numpy().view(np.uint32), n2)
    assert np.array_equal(dl.cpu().numpy().view(np.uint64), l2)
    assert np.array_equal(da.cpu().numpy().view(np.uint32), a2)
    assert np.array_equal(dp.cpu().numpy().reshape(-1, 16), p2)
    assert np.array_equal(db.cpu().numpy().reshape(-1).view(np.uint32), b2.reshape(-1).view(np.uint32))
