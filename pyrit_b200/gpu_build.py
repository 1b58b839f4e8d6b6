"""Host mirror of the reference's GPU build interface (src/gpu_build.zig) over the C ABI.

Same operations, argument meaning and error behaviour as the reference:

* :func:`build`          gpu_build.build        (src/gpu_build.zig:94-96)
* :func:`build_chunks`   gpu_build.buildChunks  (src/gpu_build.zig:119-122)
* :func:`build_chunks_edits` World.applyEdits + buildChunks as one sort-merge
                         (src/world.zig:902-1020, src/device/worldedit.zig:26-90)
* :func:`downsample`     gpu_build.downsample   (src/gpu_build.zig:128-131)
* :class:`Built`         gpu_build.Built        (src/gpu_build.zig:26-47)

Device buffers are torch CUDA tensors (plumbing only) or raw device addresses;
invalid arguments raise :class:`native.PyrbError` with result -1 (INVALID_ARGUMENT).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import native


def _addr(t) -> int:
    if t is None:
        return 0
    if isinstance(t, int):
        return t
    return int(t.data_ptr())


def _exec(stream=None) -> native.Exec:
    e = native.Exec()
    e.ctx = None
    e.stream = None if stream is None else ctypes.c_void_p(int(stream))
    return e


def _current_stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


class Built:
    """Result of a build. All buffers are device memory owned by this object (freed on
    :meth:`free` / garbage collection) -- the reference's Built.free."""

    def __init__(self, c: native.BuiltC, stream):
        self._c = c
        self._stream = stream
        self.roots = self.first_voxel = self.first_prim = None

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return getattr(self._c, name)

    def free(self):
        if self._c is not None and self._c.nodes:
            native.lib().pyrb_built_free(ctypes.byref(_exec(self._stream)), ctypes.byref(self._c))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def save_pyrd(self) -> bytes:
        """PYRD v1 bytes (pyr_geometry_download + pyr_dag_save; src/io.zig:88-129)."""
        L = native.lib()
        ex = _exec(self._stream)
        size = ctypes.c_uint64(0)
        native.check(L.pyrb_pyrd_save(ctypes.byref(ex), ctypes.byref(self._c), None, ctypes.byref(size)))
        buf = np.empty(size.value, dtype=np.uint8)
        native.check(L.pyrb_pyrd_save(ctypes.byref(ex), ctypes.byref(self._c), buf.ctypes.data, ctypes.byref(size)))
        return buf.tobytes()

    def download(self) -> "HostBuilt":
        """Copies the result to host arrays (synchronous)."""
        from . import _cudart
        c = self._c

        def fetch(addr, n, dtype):
            out = np.empty(n, dtype=dtype)
            _cudart.dtoh(out.ctypes.data, addr, out.nbytes)
            return out

        return HostBuilt(
            log2_size=c.log2_size, rt_log2=c.rt_log2, root=c.root,
            nodes=fetch(c.nodes, c.node_words, np.uint32),
            leaves=fetch(c.leaves, c.leaf_count, np.uint64),
            keys=fetch(c.keys, c.voxel_count, np.uint64),
            attrs=fetch(c.attrs, c.voxel_count, np.uint32),
            prims=fetch(c.prims, c.prim_count * 16, np.uint8),
            aabbs=fetch(c.aabbs, c.prim_count * 6, np.float32),
            roots=self.roots, first_voxel=self.first_voxel, first_prim=self.first_prim,
        )


def load_pyrd(data: bytes, stream=None) -> Built:
    """PYRD v1 bytes onto the device (pyr_dag_load, src/io.zig:131-160): nodes, leaves and
    attributes in new device buffers. Invalid data raises PyrbError (-1)."""
    stream = _current_stream() if stream is None else stream
    buf = np.frombuffer(data, dtype=np.uint8)
    out = native.BuiltC()
    native.check(native.lib().pyrb_pyrd_load(ctypes.byref(_exec(stream)), buf.ctypes.data if len(buf) else None,
                                             len(buf), ctypes.byref(out)))
    return Built(out, stream)


PALETTE_OVERFLOW = 0xFFFFFFFF


def palette_scan(attrs, first, stream=None):
    """Chunk palettes (src/device/palette.zig scan): attrs a device u32 buffer (tensor or
    address), first host uint32[count+1]. Returns (palettes: int32 CUDA tensor [count, 16]
    with the u32 values, counts: numpy uint32[count], 0xFFFFFFFF = more than 16 values)."""
    import torch
    stream = _current_stream() if stream is None else stream
    first = np.ascontiguousarray(first, dtype=np.uint32)
    count = len(first) - 1
    pal = torch.empty((max(count, 1), 16), dtype=torch.int32, device="cuda")
    counts = np.zeros(max(count, 1), dtype=np.uint32)
    native.check(native.lib().pyrb_palette_scan(ctypes.byref(_exec(stream)), _addr(attrs), first.ctypes.data, count,
                                                pal.data_ptr(), counts.ctypes.data))
    return pal[:count], counts[:count]


def palette_layout(first, counts):
    """Word offset of every chunk in the attribute pool and the pool words needed
    (palette chunks: 16 + ceil(n/8), others n; src/context.zig:1345-1352)."""
    first = np.asarray(first, dtype=np.int64)
    n = first[1:] - first[:-1]
    words = np.where(np.asarray(counts) != PALETTE_OVERFLOW, 16 + (n + 7) // 8, n)
    dst = np.concatenate([[0], np.cumsum(words)[:-1]]).astype(np.uint32) if len(words) else np.zeros(0, np.uint32)
    return dst, int(words.sum())


def palette_pack(attrs, first, palettes, counts, dst, pool, stream=None):
    """src/device/palette.zig pack into the device u32 pool at the word offsets dst."""
    stream = _current_stream() if stream is None else stream
    first = np.ascontiguousarray(first, dtype=np.uint32)
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    native.check(native.lib().pyrb_palette_pack(ctypes.byref(_exec(stream)), _addr(attrs), first.ctypes.data,
                                                len(first) - 1, _addr(palettes), counts.ctypes.data, dst.ctypes.data,
                                                _addr(pool)))


def path_edit(nodes, leaves, attributes, jobs, edits, stream=None):
    """Path edits (src/device/pathedit.zig): nodes/leaves/attributes are the device pools
    (tensors or addresses), jobs a sequence of native.PathEditJob (their out_* fields are
    filled in), edits a uint32[n, 4] host array {x, y, z, attribute} (attribute 0 removes)."""
    stream = _current_stream() if stream is None else stream
    arr = (native.PathEditJob * max(len(jobs), 1))(*jobs)
    e = np.ascontiguousarray(edits, dtype=np.uint32).reshape(-1, 4)
    native.check(native.lib().pyrb_path_edit(ctypes.byref(_exec(stream)), _addr(nodes), _addr(leaves),
                                             _addr(attributes), arr, len(jobs), e.ctypes.data if len(e) else None,
                                             len(e)))
    for i in range(len(jobs)):
        jobs[i] = arr[i]
    return jobs


@dataclass
class HostBuilt:
    log2_size: int
    rt_log2: int
    root: int
    nodes: np.ndarray
    leaves: np.ndarray
    keys: np.ndarray
    attrs: np.ndarray
    prims: np.ndarray
    aabbs: np.ndarray
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


def build(log2_size: int, rt_log2_req: int, edits=None, n_new: int | None = None, old_keys=None, old_vals=None,
          n_old: int = 0, stream=None) -> Built:
    """gpu_build.build: `edits` is a device PyrVoxel array (uint32/int32 [n, 4] tensor or address);
    `old_keys`/`old_vals` the sorted unique voxels of a previous build (copied, not consumed)."""
    if n_new is None:
        n_new = 0 if edits is None else int(edits.shape[0])
    if old_keys is not None and not isinstance(old_keys, int) and n_old == 0:
        n_old = int(old_keys.shape[0])
    stream = _current_stream() if stream is None else stream
    out = native.BuiltC()
    native.check(native.lib().pyrb_build(ctypes.byref(_exec(stream)), log2_size, rt_log2_req, _addr(old_keys),
                                         _addr(old_vals), n_old, _addr(edits), n_new, ctypes.byref(out)))
    return Built(out, stream)


def geometry_build(log2_size: int, rt_log2_req: int, voxels: np.ndarray, stream=None) -> Built:
    """pyr_geometry_build with PYR_BUILD_HOST_INPUT: host PyrVoxel array uploaded by the library."""
    v = np.ascontiguousarray(voxels, dtype=np.uint32)
    stream = _current_stream() if stream is None else stream
    out = native.BuiltC()
    native.check(native.lib().pyrb_geometry_build(ctypes.byref(_exec(stream)), log2_size, rt_log2_req,
                                                  v.ctypes.data if len(v) else None, len(v),
                                                  native.PYRB_BUILD_HOST_INPUT, ctypes.byref(out)))
    return Built(out, stream)


def build_chunks(log2_size: int, rt_log2_req: int, count: int, capacity: int, voxels, offsets, total: int,
                 stream=None) -> Built:
    """gpu_build.buildChunks: voxels device PyrVoxel[count*capacity], offsets device u32[count+1]."""
    stream = _current_stream() if stream is None else stream
    b = native.ChunkBatch(count=count, capacity=capacity, voxels=_addr(voxels), offsets=_addr(offsets), total=total)
    roots = np.zeros(count, np.uint32)
    first = np.zeros(count, np.uint32)
    prim = np.zeros(count, np.uint32)
    out = native.BuiltC()
    native.check(native.lib().pyrb_build_chunks(ctypes.byref(_exec(stream)), log2_size, rt_log2_req, ctypes.byref(b),
                                                roots.ctypes.data, first.ctypes.data, prim.ctypes.data,
                                                ctypes.byref(out)))
    r = Built(out, stream)
    r.roots, r.first_voxel, r.first_prim = roots, first, prim
    return r


def build_chunks_edits(log2_size: int, rt_log2_req: int, count: int, capacity: int, voxels, counts, edits,
                       edit_offsets, edit_total: int, stream=None) -> Built:
    """World path: generated voxels per chunk (counts) with each chunk's overlay edits merged."""
    stream = _current_stream() if stream is None else stream
    roots = np.zeros(count, np.uint32)
    first = np.zeros(count, np.uint32)
    prim = np.zeros(count, np.uint32)
    out = native.BuiltC()
    native.check(native.lib().pyrb_build_chunks_edits(
        ctypes.byref(_exec(stream)), log2_size, rt_log2_req, count, capacity, _addr(voxels), _addr(counts),
        _addr(edits), _addr(edit_offsets), edit_total, roots.ctypes.data, first.ctypes.data, prim.ctypes.data,
        ctypes.byref(out)))
    r = Built(out, stream)
    r.roots, r.first_voxel, r.first_prim = roots, first, prim
    return r


def build_batch(log2s, rt_log2_req: int, voxels, voxel_offsets, edits=None, edit_offsets=None,
                stream=None) -> Built:
    """Batched build of chunks with mixed edges (host arrays are uploaded here).

    log2s: host uint32[K]; voxels: uint32[N, 4] (chunk-local PyrVoxels, chunk c at
    voxel_offsets[c]:voxel_offsets[c+1]); optional per-chunk overlay edits. Arrays may be
    numpy (uploaded) or device tensors."""
    import torch
    stream = _current_stream() if stream is None else stream
    log2s = np.ascontiguousarray(log2s, dtype=np.uint32)
    K = len(log2s)
    keep = []

    def dev32(a):
        if a is None:
            return None
        if isinstance(a, np.ndarray):
            t = torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()
            keep.append(t)
            return t
        return a

    vo = np.asarray(voxel_offsets.cpu() if hasattr(voxel_offsets, "cpu") else voxel_offsets, dtype=np.uint32)
    eo = None if edit_offsets is None else np.asarray(
        edit_offsets.cpu() if hasattr(edit_offsets, "cpu") else edit_offsets, dtype=np.uint32)
    b = native.Batch(count=K, log2_host=log2s.ctypes.data, log2=_addr(dev32(log2s)),
                     voxels=_addr(dev32(voxels)) if int(vo[-1]) else 0, voxel_offsets=_addr(dev32(vo)),
                     edits=_addr(dev32(edits)) if eo is not None and int(eo[-1]) else 0,
                     edit_offsets=_addr(dev32(eo)) if eo is not None else 0,
                     voxel_total=int(vo[-1]), edit_total=0 if eo is None else int(eo[-1]))
    roots = np.zeros(K, np.uint32)
    first = np.zeros(K, np.uint32)
    prim = np.zeros(K, np.uint32)
    out = native.BuiltC()
    native.check(native.lib().pyrb_build_batch(ctypes.byref(_exec(stream)), ctypes.byref(b), rt_log2_req,
                                               roots.ctypes.data, first.ctypes.data, prim.ctypes.data,
                                               ctypes.byref(out)))
    r = Built(out, stream)
    r.roots, r.first_voxel, r.first_prim = roots, first, prim
    return r


def downsample(log2_src: int, rt_log2_req: int, src_keys, src_vals, n_src: int, shift: int, stream=None) -> Built:
    """gpu_build.downsample: LOD from the sorted voxels (keys/attrs) of a previous build."""
    stream = _current_stream() if stream is None else stream
    out = native.BuiltC()
    native.check(native.lib().pyrb_downsample(ctypes.byref(_exec(stream)), log2_src, rt_log2_req, _addr(src_keys),
                                              _addr(src_vals), n_src, shift, ctypes.byref(out)))
    return Built(out, stream)


def build_memory(log2_size: int, entries: int, count: int = 1, chunk_log2=None, rt_log2_req: int = 3
                 ) -> tuple[int, int]:
    """(scratch bytes, output bytes) a build of `entries` raw entries would allocate:
    one volume (count 1), `count` chunks of edge 2^log2_size, or a batch of chunks of
    edges 2^chunk_log2[c]; rt_log2_req as the build takes it. Host-only; uses the
    current tuning."""
    scratch, outs = ctypes.c_uint64(0), ctypes.c_uint64(0)
    lg = None
    if chunk_log2 is not None:
        lg = np.ascontiguousarray(chunk_log2, dtype=np.uint32)
        count = len(lg)
    native.check(native.lib().pyrb_build_memory(log2_size, rt_log2_req, count, None if lg is None else lg.ctypes.data,
                                                entries, ctypes.byref(scratch), ctypes.byref(outs)))
    return scratch.value, outs.value


def last_capacity_need() -> int:
    """Largest generator count of the last PYRB_ERROR_CAPACITY result on this thread."""
    return int(native.lib().pyrb_last_capacity_need())


def last_stats() -> native.Stats:
    s = native.Stats()
    native.lib().pyrb_last_stats(ctypes.byref(s))
    return s


def set_tuning(radix_bits: int = 0, tile_keys: int = 0, load_factor_pct: int = 50, path: int = 0) -> None:
    """Digit width and keys per sort tile (0 and 0: chosen per build, the default), the
    dedup table load factor and the path (0 automatic, 1 sort, 2 cell grid, 3 brick
    buckets), for builds started afterwards."""
    t = native.Tuning(radix_bits=radix_bits, tile_keys=tile_keys, load_factor_pct=load_factor_pct, path=path)
    native.check(native.lib().pyrb_set_tuning(ctypes.byref(t)))


def get_tuning() -> native.Tuning:
    t = native.Tuning()
    native.lib().pyrb_get_tuning(ctypes.byref(t))
    return t
