"""ctypes binding of libpyrit_b200.so (the C ABI of include/pyrit_b200.h).

There is no fallback: if the CUDA library is missing or cannot be loaded, every
entry point raises. The library is built in-tree by ``pyrit_b200._build``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpyrit_b200.so")

PYRB_OK = 0
PYRB_ERROR_INVALID_ARGUMENT = -1
PYRB_ERROR_OUT_OF_MEMORY = -3
PYRB_ERROR_CAPACITY = -4
PYRB_ERROR_CUDA = -6
PYRB_BUILD_HOST_INPUT = 0x1

ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64)
FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint64)


class Exec(ctypes.Structure):
    """pyrb_exec: stream + optional allocator callbacks (gpu_build.Exec)."""
    _fields_ = [("ctx", ctypes.c_void_p), ("stream", ctypes.c_void_p), ("alloc", ALLOC_FN), ("free", FREE_FN)]


class BuiltC(ctypes.Structure):
    """pyrb_built (gpu_build.Built, src/gpu_build.zig:26-47)."""
    _fields_ = [
        ("log2_size", ctypes.c_uint32), ("rt_log2", ctypes.c_uint32),
        ("nodes", ctypes.c_uint64), ("node_words", ctypes.c_uint32), ("root", ctypes.c_uint32),
        ("leaves", ctypes.c_uint64), ("leaf_count", ctypes.c_uint32), ("reserved0", ctypes.c_uint32),
        ("keys", ctypes.c_uint64), ("attrs", ctypes.c_uint64), ("voxel_count", ctypes.c_uint32),
        ("reserved1", ctypes.c_uint32),
        ("prims", ctypes.c_uint64), ("aabbs", ctypes.c_uint64), ("prim_count", ctypes.c_uint32),
        ("reserved2", ctypes.c_uint32),
    ]


class ChunkBatch(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint32), ("capacity", ctypes.c_uint32), ("voxels", ctypes.c_uint64),
                ("offsets", ctypes.c_uint64), ("total", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Batch(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("log2_host", ctypes.c_void_p),
                ("log2", ctypes.c_uint64), ("voxels", ctypes.c_uint64), ("voxel_offsets", ctypes.c_uint64),
                ("edits", ctypes.c_uint64), ("edit_offsets", ctypes.c_uint64), ("voxel_total", ctypes.c_uint32),
                ("edit_total", ctypes.c_uint32), ("voxel_starts", ctypes.c_uint64)]


class Stats(ctypes.Structure):
    _fields_ = [("brick_count", ctypes.c_uint32), ("level_parents", ctypes.c_uint32 * 24),
                ("level_unique", ctypes.c_uint32 * 24), ("sort_passes", ctypes.c_uint32),
                ("radix_bits", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("scratch_bytes", ctypes.c_uint64),
                ("output_bytes", ctypes.c_uint64)]


COUNTS_WORDS = 176


class Tuning(ctypes.Structure):
    _fields_ = [("radix_bits", ctypes.c_uint32), ("tile_keys", ctypes.c_uint32),
                ("load_factor_pct", ctypes.c_uint32), ("path", ctypes.c_uint32)]


PATH_AUTO, PATH_SORT, PATH_GRID, PATH_BUCKET = 0, 1, 2, 3


class ServerConfig(ctypes.Structure):
    """pyrb_server_config."""
    _fields_ = [("pool_log2", ctypes.c_void_p), ("pool_starts", ctypes.c_void_p), ("pool_sizes", ctypes.c_void_p),
                ("pool_voxels", ctypes.c_uint64), ("pool_count", ctypes.c_uint32), ("rt_log2", ctypes.c_uint32),
                ("budget_bytes", ctypes.c_uint64), ("max_batch_entries", ctypes.c_uint64),
                ("max_batch_requests", ctypes.c_uint32), ("max_edits", ctypes.c_uint32),
                ("max_inflight", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServerResult(ctypes.Structure):
    """pyrb_server_result."""
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int32), ("root", ctypes.c_uint32),
                ("first_voxel", ctypes.c_uint32), ("first_prim", ctypes.c_uint32), ("voxel_count", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("batch", BuiltC), ("latency_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    """pyrb_server_stats."""
    _fields_ = [(n, ctypes.c_uint64) for n in ("requests", "batches", "failed_batches", "evictions", "voxels",
                                               "peak_bytes", "arena_used")] + [
        (n, ctypes.c_uint32) for n in ("max_batch_requests", "pending", "inflight", "reserved")]


class PathEditJob(ctypes.Structure):
    """pyrb_path_edit_job (the reference's PathEditJob, src/device/types.zig:613-658)."""
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "node_offset", "leaf_offset", "root", "log2_size", "attr_src", "attr_count", "attr_a", "attr_b", "attr_cap",
        "palette", "pal_src", "pal_dst", "node_arena", "node_cap", "leaf_arena", "leaf_cap", "edit_first",
        "edit_count", "rt_log2", "reserved0")] + [
        ("prims", ctypes.c_uint64), ("prim_count", ctypes.c_uint32), ("reserved1", ctypes.c_uint32),
        ("aabbs", ctypes.c_uint64)] + [(n, ctypes.c_uint32) for n in (
            "aabbs_keep", "out_root", "out_count", "out_attr_b", "out_flags", "op", "op_rank", "op_attr")]


PATH_EDIT_REBUILD, PATH_EDIT_EMPTY, PATH_EDIT_OVERFLOW, PATH_EDIT_GREW = 0x1, 0x2, 0x4, 0x8

# name -> (restype, argtypes); every symbol declared in include/pyrit_b200.h
_u32, _u64, _p = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
_pu32 = ctypes.POINTER(ctypes.c_uint32)
SIGNATURES = {
    "pyrb_build": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32, _u32, _u64, _u64, _u32, _u64, _u32,
                                    ctypes.POINTER(BuiltC)]),
    "pyrb_build_chunks": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32, _u32, ctypes.POINTER(ChunkBatch), _p, _p, _p,
                                           ctypes.POINTER(BuiltC)]),
    "pyrb_build_chunks_edits": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32, _u32, _u32, _u32, _u64, _u64, _u64,
                                                 _u64, _u32, _p, _p, _p, ctypes.POINTER(BuiltC)]),
    "pyrb_downsample": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32, _u32, _u64, _u64, _u32, _u32,
                                         ctypes.POINTER(BuiltC)]),
    "pyrb_geometry_build": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32, _u32, _p, _u32, _u32,
                                             ctypes.POINTER(BuiltC)]),
    "pyrb_build_async": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32, _u32, _u64, _u64, _u32, _u64, _u32, _p,
                                          ctypes.POINTER(BuiltC)]),
    "pyrb_build_finish": (ctypes.c_int32, [_p, ctypes.POINTER(BuiltC)]),
    "pyrb_profile_enable": (None, [ctypes.c_int]),
    "pyrb_profile_read": (ctypes.c_uint32, [_p, _p, _u32, _u32]),
    "pyrb_build_batch": (ctypes.c_int32, [ctypes.POINTER(Exec), ctypes.POINTER(Batch), _u32, _p, _p, _p,
                                          ctypes.POINTER(BuiltC)]),
    "pyrb_build_batch_async": (ctypes.c_int32, [ctypes.POINTER(Exec), ctypes.POINTER(Batch), _u32, _p, _p, _p, _p,
                                                ctypes.POINTER(BuiltC)]),
    "pyrb_built_free": (None, [ctypes.POINTER(Exec), ctypes.POINTER(BuiltC)]),
    "pyrb_last_stats": (None, [ctypes.POINTER(Stats)]),
    "pyrb_error_message": (ctypes.c_char_p, []),
    "pyrb_result_string": (ctypes.c_char_p, [ctypes.c_int32]),
    "pyrb_set_tuning": (ctypes.c_int32, [ctypes.POINTER(Tuning)]),
    "pyrb_get_tuning": (None, [ctypes.POINTER(Tuning)]),
    "pyrb_version": (ctypes.c_uint32, []),
    "pyrb_pyrd_save": (ctypes.c_int32, [ctypes.POINTER(Exec), ctypes.POINTER(BuiltC), _p,
                                        ctypes.POINTER(ctypes.c_uint64)]),
    "pyrb_pyrd_load": (ctypes.c_int32, [ctypes.POINTER(Exec), _p, _u64, ctypes.POINTER(BuiltC)]),
    "pyrb_palette_scan": (ctypes.c_int32, [ctypes.POINTER(Exec), _u64, _p, _u32, _u64, _p]),
    "pyrb_path_edit": (ctypes.c_int32, [ctypes.POINTER(Exec), _u64, _u64, _u64, ctypes.POINTER(PathEditJob), _u32,
                                        _p, _u32]),
    "pyrb_palette_pack": (ctypes.c_int32, [ctypes.POINTER(Exec), _u64, _p, _u32, _u64, _p, _p, _u64]),
    "pyrb_build_noalloc": (ctypes.c_int32, [_p, _u32, _u32, _u64, _u32, _u64, _u32, _u64, _u32, _u64, _u64, _u32,
                                            _u64, _u64, _u32, ctypes.POINTER(BuiltC)]),
    "pyrb_build_memory": (ctypes.c_int32, [_u32, _u32, _u32, _p, _u64, ctypes.POINTER(ctypes.c_uint64),
                                           ctypes.POINTER(ctypes.c_uint64)]),
    "pyrb_last_capacity_need": (ctypes.c_uint32, []),
    "pyrb_selftest_wait_limit": (ctypes.c_int32, [ctypes.POINTER(Exec), _u32]),
    "pyrb_server_create": (ctypes.c_int32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "pyrb_server_submit": (ctypes.c_int32, [_p, _u64, _u32, _p, _u32]),
    "pyrb_server_poll": (ctypes.c_uint32, [_p, ctypes.POINTER(ServerResult), _u32]),
    "pyrb_server_release": (ctypes.c_int32, [_p, _u64]),
    "pyrb_server_get_stats": (None, [_p, ctypes.POINTER(ServerStats)]),
    "pyrb_server_drain": (ctypes.c_int32, [_p, _u32]),
    "pyrb_server_destroy": (None, [_p]),
}

_lib = None


class PyrbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (result {code})")
        self.code = code


def lib():
    """Loads the CUDA library; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m pyrit_b200._build` "
                               "(the DAG build has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != PYRB_OK:
        raise PyrbError(code, lib().pyrb_error_message().decode(errors="replace"))
