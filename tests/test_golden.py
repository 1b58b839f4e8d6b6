"""Committed fixtures (tests/golden/golden.json, made by tests/golden/make_golden.py):
the oracle must still produce them (CPU), and the CUDA build must reproduce them
through the C ABI (GPU): PYRD bytes of the reference GPU layout, RT prims + AABBs,
and the CPU builder's DAG after canonicalisation (src/dag_builder.zig parity)."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))
NAMES = sorted(GOLDEN)


def test_golden_covers_all_cases():
    assert sorted(make_golden.cases()) == NAMES


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    rec = make_golden.oracle_record(*make_golden.cases()[name])
    assert rec == GOLDEN[name]


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_build_matches_golden(name):
    from oracle import oracle as orc
    from pyrit_b200 import gpu_build
    from gpu_helpers import dev
    log2, rt, vox, ed = make_golden.cases()[name]
    want = GOLDEN[name]
    pts = np.concatenate([vox, ed]) if len(ed) else vox
    b = gpu_build.build(log2, rt, dev(pts))
    st = gpu_build.last_stats()
    pyrd = b.save_pyrd()
    assert hashlib.sha256(pyrd).hexdigest() == want["pyrd"]
    h = b.download()
    assert make_golden._sha(h.prims, h.aabbs) == want["prims"]
    c = want["counts"]
    assert (h.voxel_count, h.node_words, len(h.leaves), h.root, h.prim_count) == (
        c["voxel_count"], c["node_words"], c["leaf_count"], c["root"], c["prim_count"])
    assert [st.level_unique[lv] for lv in range(2, log2)] == c["level_unique"]
    gn, groot, gshared, _ = orc.canonicalize(log2, h.nodes, h.root)
    assert gshared == 0
    assert make_golden._sha(gn, np.array([groot], np.uint32), h.leaves, h.attrs) == want["canon"]
    # PYRD round trip through the device: load, save again, same bytes
    r = gpu_build.load_pyrd(pyrd)
    assert r.save_pyrd() == pyrd
    r.free()
    b.free()


@pytest.mark.gpu
def test_pyrd_load_rejects_invalid_data():
    from pyrit_b200 import gpu_build, native, workloads as wl
    from gpu_helpers import dev
    b = gpu_build.build(6, 4, dev(wl.heightfield(6, 0)))
    good = b.save_pyrd()
    b.free()
    bad = [good[:51], b"PYRX" + good[4:], good[:4] + (2).to_bytes(4, "little") + good[8:],
           good[:8] + (21).to_bytes(4, "little") + good[12:], good[:-1],
           good[:12] + (10 ** 6).to_bytes(4, "little") + good[16:]]
    for data in bad:
        with pytest.raises(native.PyrbError) as ei:
            gpu_build.load_pyrd(data)
        assert ei.value.code == -1
