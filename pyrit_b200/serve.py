"""Served chunk builds: continuous batching over a device-resident chunk pool.

The reference streams a world by building batches of chunks on a worker thread
(World.gpuWorkImpl, src/world.zig:937-1025), admitting work by its free-VRAM margin
(World.vramFree, src/world.zig:814-821) and evicting unused chunks from its pools
(src/world_plan.zig:273-292). The library's native served loop (pyrb_server_*, C++:
pyrit_b200/csrc/pyrb_server.cpp) does the same for a stream of independent chunk-build
requests:

* requests (a pool chunk plus 0..64 overlay edits) are submitted as they arrive;
* a worker thread keeps up to `max_inflight` batches on the GPU; whenever one completes,
  the requests that arrived meanwhile (up to `max_batch_voxels` voxels + edits) form the
  next batch, ONE pyrb_build_batch_async launch sequence on the server's stream --
  requests that arrive while others build join the next batch (continuous batching);
* all scratch (dedup tables, grid cells, sort buffers) and all results are sub-allocated
  from one fixed device arena of `budget_bytes` (first fit with coalescing); a batch is
  admitted when the build's exact need fits the largest free range, after evicting the
  least recently completed results;
* latency of a request = submit -> the worker saw its batch complete (host clock).

The chunk data, the dedup tables, the arena and all per-request outputs stay on the
device; this module only submits requests and collects results.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import native


@dataclass
class Request:
    rid: int
    chunk: int              # index into the pool
    edits: np.ndarray       # uint32[m, 4] chunk-local PyrVoxel overlay (attribute 0 removes)
    arrival: float          # seconds since the start of the stream


@dataclass
class RequestResult:
    batch: native.BuiltC    # buffers of the batch that built the request (server-owned)
    root: int
    first_voxel: int
    first_prim: int
    latency_ms: float


@dataclass
class ServeStats:
    requests: int = 0
    batches: int = 0
    voxels: int = 0
    duration_s: float = 0.0
    latencies_ms: list = field(default_factory=list)
    evictions: int = 0
    peak_bytes: int = 0
    max_batch_requests: int = 0

    def summary(self) -> dict:
        lat = np.array(self.latencies_ms) if self.latencies_ms else np.zeros(1)
        return {"requests": self.requests, "batches": self.batches, "voxels": self.voxels,
                "duration_s": self.duration_s, "voxels_per_s": self.voxels / max(self.duration_s, 1e-9),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "p999_ms": float(np.percentile(lat, 99.9)), "mean_ms": float(lat.mean()),
                "evictions": self.evictions, "peak_bytes": self.peak_bytes,
                "max_batch_requests": self.max_batch_requests}


class ChunkPool:
    """Device-resident chunk voxel lists (chunk c at voxels[starts[c] : starts[c] + sizes[c]])."""

    def __init__(self, voxels, offsets: np.ndarray, log2s: np.ndarray):
        self.voxels = voxels                            # int32 tensor [N, 4] on the device
        self.starts = np.asarray(offsets[:-1], dtype=np.uint64)
        self.sizes = np.diff(np.asarray(offsets, dtype=np.int64)).astype(np.uint32)
        self.log2s = np.asarray(log2s, dtype=np.uint32)

    def __len__(self):
        return len(self.log2s)


class _ArenaView:
    """Peak and current use of the server's device arena (bytes)."""

    def __init__(self, server):
        self._s = server

    @property
    def peak(self) -> int:
        return int(self._s.stats().peak_bytes)

    @property
    def used(self) -> int:
        return int(self._s.stats().arena_used)


class ChunkServer:
    """Continuous batching over a device-resident chunk pool, by the library's native
    served loop (pyrb_server_*: a worker thread, a first-fit device arena of
    `budget_bytes` for all scratch and results, admission by the build's exact memory
    need, LRU eviction). This class submits requests at their arrival times, polls the
    finished results and keeps the statistics."""

    def __init__(self, pool: ChunkPool, budget_bytes: int = 40 << 30, max_batch_voxels: int = 32 << 20,
                 max_inflight: int = 2, rt_log2: int = 5, stream=None, max_batch_requests: int = 1024,
                 max_edits_per_request: int = 64):
        self.pool = pool
        self.L = native.lib()
        self.max_edits = max_edits_per_request
        self._log2 = np.ascontiguousarray(pool.log2s, dtype=np.uint32)
        self._starts = np.ascontiguousarray(pool.starts, dtype=np.uint64)
        self._sizes = np.ascontiguousarray(pool.sizes, dtype=np.uint32)
        cfg = native.ServerConfig(pool_log2=self._log2.ctypes.data, pool_starts=self._starts.ctypes.data,
                                  pool_sizes=self._sizes.ctypes.data, pool_voxels=pool.voxels.data_ptr(),
                                  pool_count=len(self._log2), rt_log2=rt_log2, budget_bytes=budget_bytes,
                                  max_batch_entries=max_batch_voxels, max_batch_requests=max_batch_requests,
                                  max_edits=max_edits_per_request, max_inflight=max_inflight)
        h = ctypes.c_void_p()
        native.check(self.L.pyrb_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.budget = budget_bytes
        self.arena = _ArenaView(self)
        self.results: dict[int, RequestResult] = {}
        self.requests: dict[int, Request] = {}
        self.keep_results = True
        self._buf = (native.ServerResult * 4096)()

    def stats(self) -> native.ServerStats:
        st = native.ServerStats()
        self.L.pyrb_server_get_stats(self.h, ctypes.byref(st))
        return st

    def close(self):
        if self.h:
            self.L.pyrb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def release_all(self):
        for rid in list(self.results):
            self.L.pyrb_server_release(self.h, rid)
        self.results.clear()

    def _submit(self, r: Request):
        e = np.ascontiguousarray(r.edits, dtype=np.uint32).reshape(-1, 4)
        native.check(self.L.pyrb_server_submit(self.h, r.rid & 0xFFFFFFFFFFFFFFFF, r.chunk,
                                               e.ctypes.data if len(e) else None, len(e)))

    def _collect(self, stats: ServeStats) -> int:
        k = self.L.pyrb_server_poll(self.h, self._buf, len(self._buf))
        for j in range(k):
            res = self._buf[j]
            rid = int(res.id)
            rid = rid - (1 << 64) if rid >= 1 << 63 else rid
            if res.status != native.PYRB_OK:
                raise native.PyrbError(res.status, f"request {rid} failed")
            stats.latencies_ms.append(res.latency_ms)
            if self.keep_results:
                self.results[rid] = RequestResult(native.BuiltC.from_buffer_copy(res.batch), int(res.root),
                                                  int(res.first_voxel), int(res.first_prim), float(res.latency_ms))
            else:
                self.L.pyrb_server_release(self.h, res.id)
        return k

    # -- the serving loop: arrivals on the host clock, batching in the library -----
    def serve(self, requests: list[Request], realtime: bool = True) -> ServeStats:
        stats = ServeStats(requests=len(requests))
        too_many = [r.rid for r in requests if len(r.edits) > self.max_edits]
        if too_many:
            raise ValueError(f"requests {too_many[:4]} carry more than {self.max_edits} edits")
        if self.keep_results:
            for r in requests:
                self.requests[r.rid] = r
        before = self.stats()
        order = sorted(requests, key=lambda r: r.arrival)
        n, i, done = len(order), 0, 0
        t0 = time.perf_counter()
        while done < n:
            now = (time.perf_counter() - t0) if realtime else float("inf")
            while i < n and order[i].arrival <= now:
                self._submit(order[i])
                i += 1
            k = self._collect(stats)
            done += k
            if k == 0 and (i == n or not realtime):
                time.sleep(20e-6)
        stats.duration_s = time.perf_counter() - t0
        after = self.stats()
        stats.batches = int(after.batches - before.batches)
        stats.voxels = int(after.voxels - before.voxels)
        stats.evictions = int(after.evictions - before.evictions)
        stats.peak_bytes = int(after.peak_bytes)
        stats.max_batch_requests = int(after.max_batch_requests)
        return stats

    # -- access to a served result (tests) -------------------------------------
    def download(self, rid: int):
        """Host copy of the whole batch buffers holding request `rid` plus its result."""
        from .gpu_build import Built
        res = self.results[rid]
        view = Built(res.batch, None)
        host = view.download()
        view._c = None  # the server owns the buffers
        return res, host
