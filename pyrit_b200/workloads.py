"""Seeded synthetic workloads for the DAG build (ctypes over libpyrb_workloads.so).

Every generator is integer / Q16.16 fixed point, so the voxel lists are the same on
every machine. Voxels and edits are ``uint32[n, 4]`` arrays in Pyrit's PyrVoxel
layout ``{int32 x, y, z; uint32 attribute}``; attribute 0 in an edit removes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libpyrb_workloads.so")
        if not os.path.exists(path):
            from . import _build
            _build.build_workloads()
        L = ctypes.CDLL(path)
        u32, u64, p = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
        L.wl_heightfield.argtypes = [u32, u32, p, u64]
        L.wl_heightfield.restype = u64
        L.wl_noise_grid.argtypes = [u32, u32, p, u64, ctypes.POINTER(ctypes.c_int32)]
        L.wl_noise_grid.restype = u64
        L.wl_noise_edits.argtypes = [u32, u32, p, u64]
        L.wl_noise_edits.restype = u64
        L.wl_bernoulli_grid.argtypes = [u32, u32, p, u64]
        L.wl_bernoulli_grid.restype = u64
        L.wl_uniform_edits.argtypes = [u32, u64, u32, p]
        L.wl_uniform_edits.restype = u64
        L.wl_chunk_mix.argtypes = [u32, u32, p]
        L.wl_chunk_mix.restype = None
        L.wl_mix_chunk.argtypes = [u32, u32, u32, p, u64]
        L.wl_mix_chunk.restype = u64
        L.wl_chunk_edits.argtypes = [u32, u32, u32, p]
        L.wl_chunk_edits.restype = u64
        L.wl_scene_dense.argtypes = [u32, p]
        L.wl_scene_dense.restype = None
        L.wl_attr_of.argtypes = [ctypes.c_int32] * 3
        L.wl_attr_of.restype = u32
        L.wl_poisson_arrivals.argtypes = [u64, ctypes.c_double, u32, p]
        L.wl_poisson_arrivals.restype = None
        L.wl_bernoulli_at.argtypes = [u64, p, u32, p]
        L.wl_bernoulli_at.restype = None
        L.wlg_chunk_desc_bytes.restype = u64
        L.wlg_describe.argtypes = [u32, p, u32, u32, p, p, p, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.wlg_describe.restype = None
        L.wlg_heights.argtypes = [p, p, u32, u64, u32, p, p]
        L.wlg_row_counts.argtypes = [p, p, u32, u64, p, p, p]
        L.wlg_row_fill.argtypes = [p, p, u32, u64, p, p, p, p]
        _lib = L
    return _lib


def _two_phase(fn, *args):
    n = int(fn(*args, None, 0))
    out = np.empty((n, 4), dtype=np.uint32)
    if n:
        got = int(fn(*args, out.ctypes.data, n))
        assert got == n
    return out


def heightfield(log2_size: int = 6, seed: int = 0) -> np.ndarray:
    """Heightfield terrain (the 64^3 plain-build workload at log2_size 6)."""
    return _two_phase(lib().wl_heightfield, log2_size, seed)


def noise_grid(log2_size: int = 8, seed: int = 0) -> np.ndarray:
    """Thresholded 3D value noise, ~30% solid (the 256^3 workload at log2_size 8)."""
    L = lib()
    t = ctypes.c_int32()
    n = int(L.wl_noise_grid(log2_size, seed, None, 0, ctypes.byref(t)))
    out = np.empty((n, 4), dtype=np.uint32)
    if n:
        L.wl_noise_grid(log2_size, seed, out.ctypes.data, n, ctypes.byref(t))
    return out


def noise_edits(log2_size: int = 8, seed: int = 0) -> np.ndarray:
    """0.5% distinct-position set/remove edits."""
    return _two_phase(lib().wl_noise_edits, log2_size, seed)


def bernoulli_grid(log2_size: int = 10, seed: int = 0) -> np.ndarray:
    """Bernoulli(0.15) occupancy, material 1..255 (the 1024^3 worst-case dedup workload)."""
    return _two_phase(lib().wl_bernoulli_grid, log2_size, seed)


def bernoulli_at(pts: np.ndarray, seed: int = 0) -> np.ndarray:
    """Attribute of the Bernoulli grid at cells pts[n, 3] (0 = empty)."""
    pts = np.ascontiguousarray(pts, dtype=np.uint32)
    out = np.empty(len(pts), dtype=np.uint32)
    if len(pts):
        lib().wl_bernoulli_at(len(pts), pts.ctypes.data, seed, out.ctypes.data)
    return out


def uniform_edits(log2_size: int, count: int, seed: int = 0) -> np.ndarray:
    out = np.empty((count, 4), dtype=np.uint32)
    lib().wl_uniform_edits(log2_size, count, seed, out.ctypes.data)
    return out


def chunk_mix(count: int, seed: int = 0) -> np.ndarray:
    out = np.empty(count, dtype=np.uint32)
    lib().wl_chunk_mix(count, seed, out.ctypes.data)
    return out


def mix_chunk(index: int, log2: int, seed: int = 0) -> np.ndarray:
    return _two_phase(lib().wl_mix_chunk, index, log2, seed)


def chunk_edits(log2: int, count: int, seed: int = 0) -> np.ndarray:
    out = np.empty((count, 4), dtype=np.uint32)
    if count:
        lib().wl_chunk_edits(log2, count, seed, out.ctypes.data)
    return out


def scene_dense(log2_size: int) -> np.ndarray:
    """Dense test scene of the reference's tests (tests/common.zig:14-35)."""
    n = 1 << log2_size
    out = np.empty(n * n * n, dtype=np.uint32)
    lib().wl_scene_dense(log2_size, out.ctypes.data)
    return out


def dense_to_points(dense: np.ndarray, log2_size: int) -> np.ndarray:
    n = 1 << log2_size
    idx = np.nonzero(dense)[0].astype(np.uint64)
    x = idx % n
    y = (idx // n) % n
    z = idx // (n * n)
    return np.stack([x, y, z, dense[idx].astype(np.uint64)], axis=1).astype(np.uint32)


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    lib().wl_poisson_arrivals(n, rate, seed, out.ctypes.data)
    return out


def mix_chunks_device(log2s, first_index: int = 0, seed: int = 0):
    """Chunk-mix content generated on the current CUDA device (same lists as mix_chunk).

    Returns (voxels: int32 tensor [N, 4] in PyrVoxel layout, offsets: int64 numpy [K+1]).
    Chunk c is the mix chunk number first_index + c with edge 2^log2s[c]."""
    import torch
    L = lib()
    log2s = np.ascontiguousarray(log2s, dtype=np.uint32)
    K = len(log2s)
    desc = np.zeros(K * int(L.wlg_chunk_desc_bytes()), dtype=np.uint8)
    cb = np.zeros(K, np.uint64)
    rb = np.zeros(K, np.uint64)
    tc, tr = ctypes.c_uint64(), ctypes.c_uint64()
    L.wlg_describe(K, log2s.ctypes.data, first_index, seed, desc.ctypes.data, cb.ctypes.data, rb.ctypes.data,
                   ctypes.byref(tc), ctypes.byref(tr))
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    d_desc = torch.from_numpy(desc).to(dev)
    d_cb = torch.from_numpy(cb.view(np.int64)).to(dev)
    d_rb = torch.from_numpy(rb.view(np.int64)).to(dev)
    heights = torch.empty(int(tc.value), dtype=torch.int32, device=dev)
    rc = L.wlg_heights(d_desc.data_ptr(), d_cb.data_ptr(), K, tc.value, seed, heights.data_ptr(), stream)
    assert rc == 0, rc
    counts = torch.empty(int(tr.value), dtype=torch.int32, device=dev)
    rc = L.wlg_row_counts(d_desc.data_ptr(), d_rb.data_ptr(), K, tr.value, heights.data_ptr(), counts.data_ptr(),
                          stream)
    assert rc == 0, rc
    row_off = torch.cumsum(counts.to(torch.int64), 0)
    total = int(row_off[-1].item()) if len(row_off) else 0
    out = torch.empty((max(total, 1), 4), dtype=torch.int32, device=dev)
    rc = L.wlg_row_fill(d_desc.data_ptr(), d_rb.data_ptr(), K, tr.value, heights.data_ptr(), row_off.data_ptr(),
                        out.data_ptr(), stream)
    assert rc == 0, rc
    # chunk offsets: row offset at each chunk's first row
    rows_end = np.concatenate([rb[1:], [tr.value]]).astype(np.int64)
    ends = row_off[torch.from_numpy(rows_end - 1).to(dev)].cpu().numpy()
    offsets = np.concatenate([[0], ends]).astype(np.int64)
    return out[:total], offsets
