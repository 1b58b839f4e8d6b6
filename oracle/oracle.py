"""ctypes wrapper of the oracle library (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference's CPU builder (src/dag_builder.zig) and GPU
algorithm (src/device/gbuild.zig sequenced as src/gpu_build.zig) on the host. It
is the checker for the CUDA build: only tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py use it, never the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


class OrcBuilt(ctypes.Structure):
    _fields_ = [
        ("log2_size", ctypes.c_uint32), ("rt_log2", ctypes.c_uint32),
        ("nodes", ctypes.POINTER(ctypes.c_uint32)), ("node_words", ctypes.c_uint32), ("root", ctypes.c_uint32),
        ("leaves", ctypes.POINTER(ctypes.c_uint64)), ("leaf_count", ctypes.c_uint32),
        ("keys", ctypes.POINTER(ctypes.c_uint64)), ("attrs", ctypes.POINTER(ctypes.c_uint32)),
        ("voxel_count", ctypes.c_uint32),
        ("prims", ctypes.POINTER(ctypes.c_uint8)), ("aabbs", ctypes.POINTER(ctypes.c_float)),
        ("prim_count", ctypes.c_uint32),
        ("level_parents", ctypes.c_uint32 * 24), ("level_unique", ctypes.c_uint32 * 24),
        ("brick_count", ctypes.c_uint32),
    ]


class OrcDag(ctypes.Structure):
    _fields_ = [
        ("log2_size", ctypes.c_uint32), ("root", ctypes.c_uint32), ("voxel_count", ctypes.c_uint64),
        ("nodes", ctypes.POINTER(ctypes.c_uint32)), ("node_words", ctypes.c_uint64),
        ("leaves", ctypes.POINTER(ctypes.c_uint64)), ("leaf_count", ctypes.c_uint64),
        ("attrs", ctypes.POINTER(ctypes.c_uint32)), ("attr_count", ctypes.c_uint64),
    ]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        L = ctypes.CDLL(path)
        u32, u64, p = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
        L.orc_gb_build.argtypes = [u32, u32, p, p, u32, p, u32, ctypes.POINTER(OrcBuilt)]
        L.orc_gb_build_chunks.argtypes = [u32, u32, u32, u32, p, p, p, p, p, ctypes.POINTER(OrcBuilt)]
        L.orc_gb_downsample.argtypes = [u32, u32, p, p, u32, u32, ctypes.POINTER(OrcBuilt)]
        L.orc_built_free.argtypes = [ctypes.POINTER(OrcBuilt)]
        L.orc_cpu_build_points.argtypes = [u32, p, u64, ctypes.c_int, ctypes.POINTER(OrcDag)]
        L.orc_cpu_build_dense.argtypes = [u32, p, ctypes.c_int, ctypes.POINTER(OrcDag)]
        L.orc_cpu_build_overlay.argtypes = [u32, p, u64, p, u64, ctypes.c_int, ctypes.POINTER(OrcDag)]
        L.orc_cpu_build_fn_dense.argtypes = [u32, p, ctypes.c_int, ctypes.POINTER(OrcDag)]
        L.orc_dag_free.argtypes = [ctypes.POINTER(OrcDag)]
        L.orc_lookup.argtypes = [u32, p, p, p, u32, u32, u32, u32]
        L.orc_lookup.restype = u32
        L.orc_lookup_many.argtypes = [u32, p, p, p, u32, p, u64, p]
        L.orc_canonicalize.argtypes = [u32, p, u64, u32, p, u64, ctypes.POINTER(u32), ctypes.POINTER(u64), p]
        L.orc_canonicalize.restype = u64
        L.orc_rt_prims_extract.argtypes = [ctypes.POINTER(OrcDag), u32, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)),
                                           ctypes.POINTER(ctypes.POINTER(ctypes.c_float))]
        L.orc_rt_prims_extract.restype = u32
        L.orc_we_apply_all.argtypes = [u32, u32, p, p, p, p, p, p]
        L.orc_pyrd_save.argtypes = [u32, u32, u64, p, u64, p, u64, p, u64, p]
        L.orc_pyrd_save.restype = u64
        L.orc_free.argtypes = [p]
        L.orc_palette_scan.argtypes = [p, p, u32, p, p]
        L.orc_path_edit_order.argtypes = [p, u32, p]
        L.orc_path_edit.argtypes = [p, p, p, p, u32, p]
        L.orc_palette_words.argtypes = [p, u32, p, p]
        L.orc_palette_words.restype = u64
        L.orc_palette_pack.argtypes = [p, p, u32, p, p, p, p]
        _lib = L
    return _lib


def _arr(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy().view(dtype)


@dataclass
class Built:
    """Host copy of a build result in the reference GPU layout (gpu_build.Built)."""
    log2_size: int
    rt_log2: int
    nodes: np.ndarray      # uint32[node_words]
    root: int
    leaves: np.ndarray     # uint64[leaf_count]
    keys: np.ndarray       # uint64[voxel_count]
    attrs: np.ndarray      # uint32[voxel_count]
    prims: np.ndarray      # uint8[prim_count*16]
    aabbs: np.ndarray      # float32[prim_count*6]
    level_parents: list
    level_unique: list
    brick_count: int = 0
    roots: np.ndarray | None = None
    first_voxel: np.ndarray | None = None
    first_prim: np.ndarray | None = None

    @property
    def node_words(self):
        return len(self.nodes)

    @property
    def voxel_count(self):
        return len(self.attrs)

    @property
    def prim_count(self):
        return len(self.prims) // 16


def _take(b: OrcBuilt) -> Built:
    r = Built(
        log2_size=b.log2_size, rt_log2=b.rt_log2,
        nodes=_arr(b.nodes, b.node_words, np.uint32), root=b.root,
        leaves=_arr(b.leaves, b.leaf_count, np.uint64),
        keys=_arr(b.keys, b.voxel_count, np.uint64), attrs=_arr(b.attrs, b.voxel_count, np.uint32),
        prims=_arr(b.prims, b.prim_count * 16, np.uint8), aabbs=_arr(b.aabbs, b.prim_count * 6, np.float32),
        level_parents=list(b.level_parents), level_unique=list(b.level_unique), brick_count=b.brick_count,
    )
    lib().orc_built_free(ctypes.byref(b))
    return r


def _ptr(a):
    return None if a is None or len(a) == 0 else a.ctypes.data


def gb_build(log2_size, rt_log2, edits=None, old_keys=None, old_vals=None) -> Built:
    """gpu_build.build restated (src/gpu_build.zig:94)."""
    edits = np.ascontiguousarray(edits if edits is not None else np.zeros((0, 4), np.uint32), dtype=np.uint32)
    n_old = 0 if old_keys is None else len(old_keys)
    ok = None if old_keys is None else np.ascontiguousarray(old_keys, dtype=np.uint64)
    ov = None if old_vals is None else np.ascontiguousarray(old_vals, dtype=np.uint32)
    b = OrcBuilt()
    rc = lib().orc_gb_build(log2_size, rt_log2, _ptr(ok), _ptr(ov), n_old, _ptr(edits.reshape(-1)), len(edits),
                            ctypes.byref(b))
    if rc != 0:
        raise ValueError("invalid argument")
    return _take(b)


def gb_build_chunks(log2_size, rt_log2, capacity, voxels, offsets) -> Built:
    """gpu_build.buildChunks restated (src/gpu_build.zig:119). voxels: uint32[count*capacity, 4]."""
    offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
    count = len(offsets) - 1
    voxels = np.ascontiguousarray(voxels, dtype=np.uint32)
    roots = np.zeros(count, np.uint32)
    first = np.zeros(count, np.uint32)
    prim = np.zeros(count, np.uint32)
    b = OrcBuilt()
    rc = lib().orc_gb_build_chunks(log2_size, rt_log2, count, capacity, _ptr(voxels.reshape(-1)), offsets.ctypes.data,
                                   roots.ctypes.data, first.ctypes.data, prim.ctypes.data, ctypes.byref(b))
    if rc != 0:
        raise ValueError("invalid argument")
    r = _take(b)
    r.roots, r.first_voxel, r.first_prim = roots, first, prim
    return r


def gb_downsample(log2_src, rt_log2, src_keys, src_vals, shift) -> Built:
    """gpu_build.downsample restated (src/gpu_build.zig:128)."""
    sk = np.ascontiguousarray(src_keys, dtype=np.uint64)
    sv = np.ascontiguousarray(src_vals, dtype=np.uint32)
    b = OrcBuilt()
    rc = lib().orc_gb_downsample(log2_src, rt_log2, _ptr(sk), _ptr(sv), len(sk), shift, ctypes.byref(b))
    if rc != 0:
        raise ValueError("invalid argument")
    return _take(b)


@dataclass
class Dag:
    """dag_builder.Dag (src/dag_builder.zig:18-31)."""
    log2_size: int
    root: int
    voxel_count: int
    nodes: np.ndarray
    leaves: np.ndarray
    attrs: np.ndarray | None


def _take_dag(d: OrcDag) -> Dag:
    r = Dag(d.log2_size, d.root, d.voxel_count, _arr(d.nodes, d.node_words, np.uint32),
            _arr(d.leaves, d.leaf_count, np.uint64), _arr(d.attrs, d.attr_count, np.uint32) if d.attrs else None)
    lib().orc_dag_free(ctypes.byref(d))
    return r


def cpu_build_points(log2_size, points, store_attrs=True) -> Dag:
    """buildPoints restated (src/dag_builder.zig:325)."""
    pts = np.ascontiguousarray(points, dtype=np.uint32)
    d = OrcDag()
    if lib().orc_cpu_build_points(log2_size, _ptr(pts.reshape(-1)), len(pts), int(store_attrs), ctypes.byref(d)) != 0:
        raise ValueError("invalid argument")
    return _take_dag(d)


def cpu_build_overlay(log2_size, voxels, edits, store_attrs=True) -> Dag:
    """Edits merged by a host hash map, then buildPoints (tests/cpu_test.zig:829-838)."""
    v = np.ascontiguousarray(voxels, dtype=np.uint32)
    e = np.ascontiguousarray(edits, dtype=np.uint32)
    d = OrcDag()
    if lib().orc_cpu_build_overlay(log2_size, _ptr(v.reshape(-1)), len(v), _ptr(e.reshape(-1)), len(e),
                                   int(store_attrs), ctypes.byref(d)) != 0:
        raise ValueError("invalid argument")
    return _take_dag(d)


def cpu_build_dense(log2_size, dense, store_attrs=True) -> Dag:
    """buildDense restated (src/dag_builder.zig:292)."""
    v = np.ascontiguousarray(dense, dtype=np.uint32)
    d = OrcDag()
    if lib().orc_cpu_build_dense(log2_size, v.ctypes.data, int(store_attrs), ctypes.byref(d)) != 0:
        raise ValueError("invalid argument")
    return _take_dag(d)


def cpu_build_fn_dense(log2_size, dense, store_attrs=True) -> Dag:
    """buildFn restated over a dense table (src/dag_builder.zig:373)."""
    v = np.ascontiguousarray(dense, dtype=np.uint32)
    d = OrcDag()
    if lib().orc_cpu_build_fn_dense(log2_size, v.ctypes.data, int(store_attrs), ctypes.byref(d)) != 0:
        raise ValueError("invalid argument")
    return _take_dag(d)


def lookup_many(log2_size, nodes, leaves, attrs, root, pts) -> np.ndarray:
    """Dag.lookup restated (src/dag_builder.zig:35-61) over many points; 0 = empty."""
    pts = np.ascontiguousarray(pts, dtype=np.uint32)
    out = np.zeros(len(pts), dtype=np.uint32)
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    leaves = np.ascontiguousarray(leaves, dtype=np.uint64)
    attrs = None if attrs is None else np.ascontiguousarray(attrs, dtype=np.uint32)
    lib().orc_lookup_many(log2_size, nodes.ctypes.data, _ptr(leaves), _ptr(attrs), root, _ptr(pts.reshape(-1)),
                          len(pts), out.ctypes.data)
    return out


def canonicalize(log2_size, nodes, root):
    """Level-order relabelling: returns (canonical nodes, canonical root, shared_across_levels, level_unique)."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    L = lib()
    r = ctypes.c_uint32()
    sh = ctypes.c_uint64()
    lu = (ctypes.c_uint32 * 24)()
    w = int(L.orc_canonicalize(log2_size, nodes.ctypes.data, len(nodes), root, None, 0, ctypes.byref(r),
                               ctypes.byref(sh), lu))
    out = np.zeros(max(w, 1), dtype=np.uint32)
    L.orc_canonicalize(log2_size, nodes.ctypes.data, len(nodes), root, out.ctypes.data, w, ctypes.byref(r),
                       ctypes.byref(sh), None)
    return out[:w], int(r.value), int(sh.value), list(lu)


def rt_prims_extract(dag: Dag, requested_log2: int):
    """rt_prims.extract restated (src/rt_prims.zig:123): (prims uint8[n*16], aabbs float32[n*6])."""
    d = OrcDag()
    d.log2_size, d.root, d.voxel_count = dag.log2_size, dag.root, dag.voxel_count
    d.nodes = dag.nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    d.node_words = len(dag.nodes)
    d.leaves = dag.leaves.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
    d.leaf_count = len(dag.leaves)
    pp = ctypes.POINTER(ctypes.c_uint8)()
    ap = ctypes.POINTER(ctypes.c_float)()
    L = lib()
    n = L.orc_rt_prims_extract(ctypes.byref(d), requested_log2, ctypes.byref(pp), ctypes.byref(ap))
    prims = _arr(pp, n * 16, np.uint8)
    aabbs = _arr(ap, n * 6, np.float32)
    L.orc_free(ctypes.cast(pp, ctypes.c_void_p))
    L.orc_free(ctypes.cast(ap, ctypes.c_void_p))
    return prims, aabbs


def we_apply_all(count, capacity, voxels, counts, edits, edit_offsets):
    """worldedit apply/compact/append restated (src/device/worldedit.zig:26-90)."""
    v = np.ascontiguousarray(voxels, dtype=np.uint32).copy()
    c = np.ascontiguousarray(counts, dtype=np.uint32)
    e = np.ascontiguousarray(edits, dtype=np.uint32)
    eo = np.ascontiguousarray(edit_offsets, dtype=np.uint32)
    ov = np.zeros_like(v)
    oc = np.zeros(count, np.uint32)
    lib().orc_we_apply_all(count, capacity, _ptr(v.reshape(-1)), c.ctypes.data, _ptr(e.reshape(-1)), eo.ctypes.data,
                           _ptr(ov.reshape(-1)), oc.ctypes.data)
    return ov, oc


def pyrd_bytes(log2_size, root, voxel_count, nodes, leaves, attrs) -> bytes:
    """PYRD v1 byte stream (src/io.zig:88-129)."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
    leaves = np.ascontiguousarray(leaves, dtype=np.uint64)
    a = None if attrs is None else np.ascontiguousarray(attrs, dtype=np.uint32)
    L = lib()
    args = (log2_size, root, voxel_count, nodes.ctypes.data, len(nodes), _ptr(leaves), len(leaves), _ptr(a),
            0 if a is None else len(a))
    n = int(L.orc_pyrd_save(*args, None))
    buf = np.zeros(n, dtype=np.uint8)
    L.orc_pyrd_save(*args, buf.ctypes.data)
    return buf.tobytes()


def morton(x, y, z) -> int:
    def spread(v):
        r = 0
        for i in range(21):
            r |= ((v >> i) & 1) << (3 * i)
        return r
    return spread(x) | (spread(y) << 1) | (spread(z) << 2)


def local_key(x, y, z) -> int:
    """Voxel key: (brick Morton << 6) | x&3 + 4(y&3) + 16(z&3) (src/device/gbuild.zig:98-101)."""
    return (morton(x >> 2, y >> 2, z >> 2) << 6) | ((x & 3) + 4 * (y & 3) + 16 * (z & 3))


def palette_scan(attrs, first):
    """palette.zig scan (src/device/palette.zig:55-104), chunks one after the other:
    returns (palettes uint32[count, 16], counts uint32[count]; 0xFFFFFFFF = overflow)."""
    attrs = np.ascontiguousarray(attrs, dtype=np.uint32)
    first = np.ascontiguousarray(first, dtype=np.uint32)
    count = len(first) - 1
    pal = np.zeros((max(count, 1), 16), dtype=np.uint32)
    counts = np.zeros(max(count, 1), dtype=np.uint32)
    lib().orc_palette_scan(_ptr(attrs), first.ctypes.data, count, pal.ctypes.data, counts.ctypes.data)
    return pal[:count], counts[:count]


def palette_layout(first, counts):
    """Word offset of every chunk in the attribute pool and the total (src/context.zig:1345-1352)."""
    first = np.ascontiguousarray(first, dtype=np.uint32)
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    dst = np.zeros(max(len(counts), 1), dtype=np.uint32)
    total = int(lib().orc_palette_words(first.ctypes.data, len(counts), counts.ctypes.data, dst.ctypes.data))
    return dst[:len(counts)], total


def palette_pack(attrs, first, palettes, counts, dst, total_words):
    """palette.zig pack (src/device/palette.zig:107-152) into a fresh pool of total_words."""
    attrs = np.ascontiguousarray(attrs, dtype=np.uint32)
    first = np.ascontiguousarray(first, dtype=np.uint32)
    pool = np.zeros(max(total_words, 1), dtype=np.uint32)
    lib().orc_palette_pack(_ptr(attrs), first.ctypes.data, len(counts), np.ascontiguousarray(palettes).ctypes.data,
                           np.ascontiguousarray(counts, dtype=np.uint32).ctypes.data,
                           np.ascontiguousarray(dst, dtype=np.uint32).ctypes.data, pool.ctypes.data)
    return pool[:total_words]


class OrcPathEditJob(ctypes.Structure):
    """orc_path_edit_job (the reference's PathEditJob, src/device/types.zig:613-658)."""
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "node_offset", "leaf_offset", "root", "log2_size", "attr_src", "attr_count", "attr_a", "attr_b", "attr_cap",
        "palette", "pal_src", "pal_dst", "node_arena", "node_cap", "leaf_arena", "leaf_cap", "edit_first",
        "edit_count", "rt_log2", "reserved0")] + [
        ("prims", ctypes.c_uint64), ("prim_count", ctypes.c_uint32), ("reserved1", ctypes.c_uint32),
        ("aabbs", ctypes.c_uint64)] + [(n, ctypes.c_uint32) for n in (
            "aabbs_keep", "out_root", "out_count", "out_attr_b", "out_flags", "op", "op_rank", "op_attr")]


def path_edit(nodes, leaves, attrs, jobs, edits, prims=None, aabbs=None):
    """pathedit.zig restated: edits each job in place on host copies of the pools.
    jobs: list of dicts of job fields (prims/aabbs are taken as the given host arrays,
    shared by all jobs with prim offsets in 'prim_first'). Returns (nodes, leaves, attrs,
    prims, aabbs, jobs as dicts with the out_* fields)."""
    nodes = np.array(nodes, dtype=np.uint32)
    leaves = np.array(leaves, dtype=np.uint64)
    attrs = np.array(attrs, dtype=np.uint32)
    prims = None if prims is None else np.array(prims, dtype=np.uint8).reshape(-1, 16)
    aabbs = None if aabbs is None else np.array(aabbs, dtype=np.float32).reshape(-1, 6)
    e = np.array(edits, dtype=np.uint32).reshape(-1, 4)
    arr = (OrcPathEditJob * max(len(jobs), 1))()
    for i, jd in enumerate(jobs):
        for k, v in jd.items():
            if k in ("prim_first",):
                continue
            setattr(arr[i], k, v)
        pf = jd.get("prim_first", 0)
        arr[i].prims = 0 if prims is None or jd.get("prim_count", 0) == 0 else prims.ctypes.data + 16 * pf
        arr[i].aabbs = 0 if aabbs is None or jd.get("prim_count", 0) == 0 else aabbs.ctypes.data + 24 * pf
    L = lib()
    L.orc_path_edit_order(arr, len(jobs), e.ctypes.data)
    L.orc_path_edit(nodes.ctypes.data, leaves.ctypes.data, attrs.ctypes.data, arr, len(jobs), e.ctypes.data)
    out = [{f: getattr(arr[i], f) for f, _ in OrcPathEditJob._fields_} for i in range(len(jobs))]
    return nodes, leaves, attrs, prims, aabbs, out
