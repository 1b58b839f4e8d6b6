"""pyrb_build_noalloc: the build variant for callers that cannot allocate device memory
while they build (frame loops that must not synchronise the device through
cudaMalloc, code running during CUDA graph stream capture, fixed memory budgets).
It keeps all scratch in a fixed device array inside the library; the test allocates
the input and output buffers itself and checks, over two calls in a row, that the
results equal pyrb_build's bit for bit (the second call also shows that the shared
array is cleared between calls). This file is collected last on purpose."""
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
