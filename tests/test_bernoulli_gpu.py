"""Worst-case dedup workload: i.i.d. Bernoulli(0.15) occupancy with materials 1..255 and
uniform set/remove edits. Exact parity with the oracle at 256^3; at the full 1024^3
(2^30 cells, ~1.6e8 voxels, 10^6 edits) size-independent properties: sorted unique keys,
point lookups through the built DAG equal the generator's definition with the edits
applied (last one wins), counts consistent across levels."""
import numpy as np
import pytest

from oracle import oracle as orc
from pyrit_b200 import workloads as wl

from gpu_helpers import assert_same_build, dev

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["sort", "grid", "bucket"])
def path(request):
    """The sparse worst case on every path: the radix sort (the automatic choice at 6.6
    cells per entry), the cell grid and the brick buckets forced."""
    from pyrit_b200 import gpu_build, native
    gpu_build.set_tuning(0, 0, 50, {"sort": native.PATH_SORT, "grid": native.PATH_GRID,
                                    "bucket": native.PATH_BUCKET}[request.param])
    yield request.param
    gpu_build.set_tuning(0, 0, 50, native.PATH_AUTO)


def test_bernoulli_256_matches_oracle(path):
    from pyrit_b200 import gpu_build
    vox = wl.bernoulli_grid(8, 1)
    ed = wl.uniform_edits(8, 16000, 1)
    pts = np.concatenate([vox, ed])
    g = gpu_build.build(8, 5, dev(pts)).download()
    assert_same_build(g, orc.gb_build(8, 5, pts), label="bernoulli256 " + path)


def test_bernoulli_1024_properties(path):
    import torch
    from pyrit_b200 import gpu_build
    log2, seed = 10, 0
    vox = wl.bernoulli_grid(log2, seed)
    ed = wl.uniform_edits(log2, 1_000_000, seed)
    pts = np.concatenate([vox, ed])
    del vox
    b = gpu_build.build(log2, 7, dev(pts))
    st = gpu_build.last_stats()
    # the memory the build took is the host-side bound, under the reference's 130 B/voxel
    scratch, outputs = gpu_build.build_memory(log2, len(pts), rt_log2_req=7)
    assert (st.scratch_bytes, st.output_bytes) == (scratch, outputs)
    assert (scratch + outputs) / len(pts) < 130
    h = b.download()
    b.free()
    torch.cuda.empty_cache()
    k = h.keys
    assert len(k) == h.voxel_count and np.all(k[1:] > k[:-1])
    assert int(h.nodes[h.root + 1]) == h.voxel_count
    # lookups: random cells plus every edited cell
    rng = np.random.default_rng(1)
    sample = np.concatenate([rng.integers(0, 1 << log2, (200_000, 3)).astype(np.uint32), ed[:, :3]])
    got = orc.lookup_many(log2, h.nodes, h.leaves, h.attrs, h.root, sample)
    want = wl.bernoulli_at(sample, seed)
    last = {}
    for i, (x, y, z, a) in enumerate(ed.tolist()):
        last[(x, y, z)] = a
    for i, (x, y, z) in enumerate(sample.tolist()):
        a = last.get((x, y, z))
        if a is not None:
            want[i] = a
    assert np.array_equal(got, want)
    # per-level counts: every level has parents, unique <= parents
    for lv in range(2, log2):
        assert 0 < st.level_unique[lv] <= st.level_parents[lv]


@pytest.mark.slow
def test_bernoulli_1024_equals_cpu_builder():
    """Full size against the reference's CPU builder (hash-map merge + buildPoints,
    src/dag_builder.zig): node count per level, canonical node/pointer buffer, root,
    leaves and attributes equal."""
    import torch
    from pyrit_b200 import gpu_build
    log2, seed = 10, 0
    vox = wl.bernoulli_grid(log2, seed)
    ed = wl.uniform_edits(log2, 1_000_000, seed)
    b = gpu_build.build(log2, 7, dev(np.concatenate([vox, ed])))
    st = gpu_build.last_stats()
    g = b.download()
    b.free()
    torch.cuda.empty_cache()
    ref = orc.cpu_build_overlay(log2, vox, ed)
    del vox
    assert g.voxel_count == ref.voxel_count
    assert np.array_equal(g.attrs, ref.attrs)
    assert np.array_equal(g.leaves, ref.leaves)
    cn, croot, shared, lu = orc.canonicalize(log2, ref.nodes, ref.root)
    gn, groot, gshared, glu = orc.canonicalize(log2, g.nodes, g.root)
    assert gshared == 0 and shared == 0
    assert list(lu) == list(glu)
    for lv in range(2, log2):
        assert st.level_unique[lv] == lu[lv], (lv, st.level_unique[lv], lu[lv])
    assert np.array_equal(gn, g.nodes) and groot == g.root
    assert np.array_equal(cn, gn) and croot == groot
