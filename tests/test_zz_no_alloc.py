"""pyrb_build_noalloc: the build variant for callers that cannot allocate device memory
while they build -- a render or frame loop must not call cudaMalloc, which synchronises
the whole device, and an engine with a fixed memory budget has no allocator to hand over.
It keeps all scratch in a fixed device array inside the library; the test allocates
the input and output buffers itself and checks, over two calls in a row, that the
results equal pyrb_build's bit for bit (the second call also shows that the shared
array is cleared between calls), and at the documented limit (edge 256, about 2^20
voxels) that they equal the oracle's. This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from pyrit_b200 import workloads as wl

from gpu_helpers import dev

pytestmark = pytest.mark.gpu


def _bounds(log2, rt, n):
    """Output sizes the build needs (the same upper bounds the library uses)."""
    nmax = max(n, 1)
    B = max(min(nmax, 8 ** (log2 - 2)), 1)
    P, words, prev = {}, 2, B
    for lv in range(2, log2):
        P[lv] = max(min(prev, 8 ** (log2 - lv - 1)), 1)
        prev = P[lv]
        words += 10 * P[lv]
    rt = min(max(rt, 3), log2)
    return words, B, nmax, max(P[rt - 1], 1)


def _noalloc_build(log2, rt, pts):
    import torch
    from pyrit_b200 import native
    n = len(pts)
    words, leaves_n, vox_n, prim_n = _bounds(log2, rt, n)
    nodes = torch.zeros(words, dtype=torch.int32, device="cuda")
    leaves = torch.zeros(leaves_n, dtype=torch.int64, device="cuda")
    keys = torch.zeros(vox_n, dtype=torch.int64, device="cuda")
    attrs = torch.zeros(vox_n, dtype=torch.int32, device="cuda")
    prims = torch.zeros(prim_n * 4, dtype=torch.int32, device="cuda")
    aabbs = torch.zeros(prim_n * 6, dtype=torch.float32, device="cuda")
    inp = dev(pts)
    out = native.BuiltC()
    stream = torch.cuda.current_stream().cuda_stream
    native.check(native.lib().pyrb_build_noalloc(
        ctypes.c_void_p(stream), log2, rt, 0 if inp is None else inp.data_ptr(), n,
        nodes.data_ptr(), words, leaves.data_ptr(), leaves_n, keys.data_ptr(), attrs.data_ptr(), vox_n,
        prims.data_ptr(), aabbs.data_ptr(), prim_n, ctypes.byref(out)))
    torch.cuda.synchronize()
    return {
        "node_words": out.node_words, "root": out.root, "leaf_count": out.leaf_count,
        "voxel_count": out.voxel_count, "prim_count": out.prim_count,
        "nodes": nodes.cpu().numpy().view(np.uint32)[:out.node_words],
        "leaves": leaves.cpu().numpy().view(np.uint64)[:out.leaf_count],
        "keys": keys.cpu().numpy().view(np.uint64)[:out.voxel_count],
        "attrs": attrs.cpu().numpy().view(np.uint32)[:out.voxel_count],
        "prims": prims.cpu().numpy().view(np.uint8)[:out.prim_count * 16],
        "aabbs": aabbs.cpu().numpy().view(np.uint32)[:out.prim_count * 6],
    }


def _scene(log2):
    pts = wl.dense_to_points(wl.scene_dense(log2), log2)
    np.random.default_rng(21).shuffle(pts)
    return np.concatenate([pts, pts[:200], np.array([[0xFFFFFFFF, 0, 0, 5], [1 << log2, 0, 0, 5]], np.uint32)])


def test_noalloc_matches_pyrb_build_two_calls_in_a_row():
    import torch
    assert torch.cuda.is_available()
    from pyrit_b200 import gpu_build
    cases = [(6, 4, wl.heightfield(6, 0)), (6, 4, _scene(6))]
    for log2, rt, pts in cases:
        got = _noalloc_build(log2, rt, pts)
        ref = gpu_build.build(log2, rt, dev(pts), n_new=len(pts)).download()
        for f in ("node_words", "root", "voxel_count", "prim_count"):
            assert got[f] == getattr(ref, f), f
        assert got["leaf_count"] == len(ref.leaves)
        assert np.array_equal(got["nodes"], ref.nodes)
        assert np.array_equal(got["leaves"], ref.leaves)
        assert np.array_equal(got["keys"], ref.keys)
        assert np.array_equal(got["attrs"], ref.attrs)
        assert np.array_equal(got["prims"], ref.prims)
        assert np.array_equal(got["aabbs"], ref.aabbs.view(np.uint32))


def _noise_octant_near_limit():
    """About 10^6 entries at edge 256: the noise grid and its edits inside the octant
    [0, 128)^3, plus repeats of part of it with new attributes (the last one wins)."""
    vox, ed = wl.noise_grid(8, 0), wl.noise_edits(8, 0)
    inside = lambda p: p[(p[:, 0] < 128) & (p[:, 1] < 128) & (p[:, 2] < 128)]
    base = np.concatenate([inside(vox), inside(ed)])
    rng = np.random.default_rng(4)
    rep = base[rng.integers(0, len(base), (1 << 20) - 2 - len(base))].copy()
    rep[:, 3] = rng.integers(0, 9, len(rep))
    pts = np.concatenate([base, rep, np.array([[300, 0, 0, 7], [0, 0xFFFFFFFF, 0, 7]], np.uint32)])
    assert len(pts) == 1 << 20
    return pts


def test_noalloc_at_its_limit_matches_the_oracle_two_calls_in_a_row():
    from oracle import oracle as orc
    pts = _noise_octant_near_limit()
    o = orc.gb_build(8, 5, pts)
    for _ in range(2):
        got = _noalloc_build(8, 5, pts)
        assert got["voxel_count"] == o.voxel_count and got["node_words"] == o.node_words
        assert got["root"] == o.root and got["prim_count"] == o.prim_count
        assert np.array_equal(got["nodes"], o.nodes)
        assert np.array_equal(got["leaves"], o.leaves)
        assert np.array_equal(got["keys"], o.keys)
        assert np.array_equal(got["attrs"], o.attrs)
        assert np.array_equal(got["prims"], o.prims)
        assert np.array_equal(got["aabbs"], o.aabbs.view(np.uint32))


def test_noalloc_without_input_builds_the_empty_geometry():
    from pyrit_b200 import gpu_build
    got = _noalloc_build(5, 3, np.zeros((0, 4), np.uint32))  # n_new 0, edits NULL
    ref = gpu_build.build(5, 3, None, n_new=0).download()
    assert got["voxel_count"] == 0 and got["node_words"] == ref.node_words == 2
    assert got["root"] == ref.root and np.array_equal(got["nodes"], ref.nodes)


def test_noalloc_rejects_sizes_beyond_its_limit():
    from pyrit_b200 import native
    out = native.BuiltC()
    L = native.lib()
    # edge 512 exceeds the fixed limit (log2_size <= 8): rejected before any GPU work
    rc = L.pyrb_build_noalloc(None, 9, 3, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, ctypes.byref(out))
    assert rc == native.PYRB_ERROR_INVALID_ARGUMENT
    assert b"log2_size" in L.pyrb_error_message()
    rc = L.pyrb_build_noalloc(None, 6, 3, 1, (1 << 20) + 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, ctypes.byref(out))
    assert rc == native.PYRB_ERROR_INVALID_ARGUMENT
    assert b"limit" in L.pyrb_error_message()
