"""Helpers shared by the GPU parity tests: device upload and byte-exact comparison
of a CUDA build against the oracle's restatement of the reference GPU algorithm."""
from __future__ import annotations

import numpy as np


def dev(a: np.ndarray):
    """numpy uint32/uint64 array -> torch CUDA tensor with the same bytes (None if empty)."""
    import torch
    if a is None or a.size == 0:
        return None
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        t = torch.from_numpy(a.view(np.int32))
    elif a.dtype == np.uint64:
        t = torch.from_numpy(a.view(np.int64))
    else:
        t = torch.from_numpy(a)
    return t.cuda()


def assert_same_build(g, o, chunks: bool = False, label: str = ""):
    """g: pyrit_b200 HostBuilt, o: oracle Built. Bit-exact on every output buffer."""
    assert g.voxel_count == o.voxel_count, f"{label} voxel_count {g.voxel_count} != {o.voxel_count}"
    assert np.array_equal(g.keys, o.keys), f"{label} keys differ"
    assert np.array_equal(g.attrs, o.attrs), f"{label} attrs differ"
    assert g.leaves.shape == o.leaves.shape, f"{label} leaf_count {len(g.leaves)} != {len(o.leaves)}"
    assert np.array_equal(g.leaves, o.leaves), f"{label} leaves differ"
    assert g.node_words == o.node_words, f"{label} node_words {g.node_words} != {o.node_words}"
    if not np.array_equal(g.nodes, o.nodes):
        bad = np.nonzero(g.nodes != o.nodes)[0]
        raise AssertionError(f"{label} nodes differ at {bad[:8]} (of {len(bad)})")
    assert g.root == o.root, f"{label} root {g.root} != {o.root}"
    assert g.prim_count == o.prim_count, f"{label} prim_count {g.prim_count} != {o.prim_count}"
    assert np.array_equal(g.prims, o.prims), f"{label} prims differ"
    assert np.array_equal(g.aabbs.view(np.uint32), o.aabbs.view(np.uint32)), f"{label} aabbs differ"
    if chunks:
        assert np.array_equal(g.roots, o.roots), f"{label} roots differ"
        assert np.array_equal(g.first_voxel, o.first_voxel), f"{label} first_voxel differ"
        assert np.array_equal(g.first_prim, o.first_prim), f"{label} first_prim differ"


def subdag(log2, nodes, leaves, root):
    """Canonical form of the DAG below `root`: nodes level by level (8^3 level first,
    first visit in child-index order), leaves renumbered by first visit. Returns
    (node words, leaf masks, root offset). Lets a chunk of a shared batch buffer be
    compared with its own single build."""
    top = log2 - 1
    order = {lv: [] for lv in range(2, top + 1)}
    seen = {lv: {} for lv in range(2, top + 1)}
    leaf_ids, leaf_list = {}, []
    seen[top][int(root)] = 0
    order[top].append(int(root))
    # iterative DFS with explicit child order
    visit = [(int(root), top, 0)]
    while visit:
        off, lv, k = visit.pop()
        n = bin(int(nodes[off]) & 0xFF).count("1")
        if k >= n:
            continue
        visit.append((off, lv, k + 1))
        ref = int(nodes[off + 2 + k])
        if lv == 2:
            if ref not in leaf_ids:
                leaf_ids[ref] = len(leaf_list)
                leaf_list.append(int(leaves[ref]))
        elif ref not in seen[lv - 1]:
            seen[lv - 1][ref] = len(order[lv - 1])
            order[lv - 1].append(ref)
            visit.append((ref, lv - 1, 0))
    coff, w = {}, 0
    for lv in range(2, top + 1):
        for off in order[lv]:
            coff[(lv, off)] = w
            w += 2 + bin(int(nodes[off]) & 0xFF).count("1")
    out = []
    for lv in range(2, top + 1):
        for off in order[lv]:
            n = bin(int(nodes[off]) & 0xFF).count("1")
            out += [int(nodes[off]), int(nodes[off + 1])]
            for k in range(n):
                ref = int(nodes[off + 2 + k])
                out.append(leaf_ids[ref] if lv == 2 else coff[(lv - 1, ref)])
    return out, leaf_list, coff[(top, int(root))]
