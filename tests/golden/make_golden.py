"""Generates tests/golden/golden.json: SHA-256 digests of the oracle's outputs on the
seeded workloads, the fixtures that the CPU tests (oracle vs fixture) and the GPU
parity tests (CUDA build vs fixture) check against.

The reference (Zig 0.16) cannot be built or imported here, so the fixtures are
outputs of the oracle, whose restatement is pinned to the reference's own
known-answer tests (tests/test_oracle.py). Each case records:

  pyrd      sha256 of the PYRD v1 bytes (src/io.zig:88-129) of the build in the
            reference GPU layout (gbuild.zig ops sequenced as gpu_build.buildImpl)
  prims     sha256 of the RT prims (16 B each) followed by the AABBs (f32 x 6)
  canon     sha256 of the CPU builder's DAG (src/dag_builder.zig; edits merged by a
            hash map first) after level-order canonicalisation: canonical node
            words, leaves, attributes
  counts    voxel_count, node_words, leaf_count, root, prim_count, unique nodes per level

Run: python tests/golden/make_golden.py   (rewrites golden.json)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def cases():
    """name -> (log2_size, rt_log2, voxels uint32[n,4], edits uint32[m,4])."""
    from pyrit_b200 import workloads as wl
    out = {}
    out["heightfield64"] = (6, 4, wl.heightfield(6, 0), np.zeros((0, 4), np.uint32))
    out["scene64"] = (6, 4, wl.dense_to_points(wl.scene_dense(6), 6), np.zeros((0, 4), np.uint32))
    out["noise256_edits"] = (8, 7, wl.noise_grid(8, 0), wl.noise_edits(8, 0))
    out["bernoulli128_edits"] = (7, 5, wl.bernoulli_grid(7, 3), wl.uniform_edits(7, 20000, 3))
    out["mixchunk_c7_e128"] = (7, 5, wl.mix_chunk(7, 7, 0), wl.chunk_edits(7, 64, 1))
    return out


def digest_pyrd(pyrd: bytes) -> str:
    return hashlib.sha256(pyrd).hexdigest()


def oracle_record(log2, rt, vox, ed):
    from oracle import oracle as orc
    pts = np.concatenate([vox, ed]) if len(ed) else vox
    g = orc.gb_build(log2, rt, pts)
    pyrd = orc.pyrd_bytes(log2, g.root, int(g.nodes[g.root + 1]), g.nodes, g.leaves, g.attrs)
    ref = orc.cpu_build_overlay(log2, vox, ed)
    cn, croot, shared, lu = orc.canonicalize(log2, ref.nodes, ref.root)
    return {
        "pyrd": digest_pyrd(pyrd),
        "prims": _sha(g.prims, g.aabbs),
        "canon": _sha(cn, np.array([croot], np.uint32), ref.leaves, ref.attrs),
        "counts": {"voxel_count": int(g.voxel_count), "node_words": int(len(g.nodes)), "leaf_count": int(len(g.leaves)),
                   "root": int(g.root), "prim_count": int(g.prim_count),
                   "level_unique": [int(x) for x in lu[2:log2]], "cpu_shared_across_levels": int(shared)},
    }


def main():
    res = {name: oracle_record(*c) for name, c in cases().items()}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)
        f.write("\n")
    print(json.dumps({k: v["counts"] for k, v in res.items()}, indent=1))


if __name__ == "__main__":
    main()
