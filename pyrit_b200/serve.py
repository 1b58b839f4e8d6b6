"""Served chunk builds: continuous batching over a device-resident chunk pool.

The reference streams a world by building batches of chunks on a worker thread
(World.gpuWorkImpl, src/world.zig:937-1025), admitting work by its free-VRAM margin
(World.vramFree, src/world.zig:814-821) and evicting unused chunks from its pools
(src/world_plan.zig:273-292). This is the same loop for a stream of independent
chunk-build requests:

* requests (a pool chunk plus 0..64 overlay edits) arrive over time;
* whenever fewer than `max_inflight` batches are on the GPU, every pending request
  (up to `max_batch_voxels`) forms the next batch, which is ONE pyrb_build_batch_async
  launch sequence on the server's stream -- requests that arrive while others build
  join the next batch (continuous batching);
* admission is by memory accounting: a batch is launched only when its scratch and
  output bound fit into `budget_bytes` next to the resident results; the least
  recently used resident batches are evicted first;
* latency of a request = device completion time of its batch (CUDA events on the
  server stream, relative to an event at t=0) minus its arrival time.

The chunk data, the dedup tables, the node/leaf/attribute arena and all per-request
outputs stay on the device; the host only forms batches and reads counts.
"""
from __future__ import annotations

import collections
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
    batch: int
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


class _Batch:
    def __init__(self, bid, reqs, built, done, keep, roots, first, fprim, counts, entries, reserve):
        self.bid, self.reqs, self.built, self.done, self.keep = bid, reqs, built, done, keep
        self.roots, self.first, self.fprim, self.counts = roots, first, fprim, counts
        self.entries, self.reserve, self.bytes = entries, reserve, reserve


class ChunkServer:
    # scratch + output bound per entry of a batch build (sort buffers, unique keys and
    # attributes, bricks, dedup tables, node bound), a safe over-estimate
    BYTES_PER_ENTRY = 96
    BYTES_FIXED = 64 << 20

    def __init__(self, pool: ChunkPool, budget_bytes: int = 40 << 30, max_batch_voxels: int = 128 << 20,
                 max_inflight: int = 2, rt_log2: int = 5, stream=None):
        import torch
        self.pool = pool
        self.budget = budget_bytes
        self.max_batch_voxels = max_batch_voxels
        self.max_inflight = max_inflight
        self.rt = rt_log2
        self.stream = stream or torch.cuda.Stream()
        self.ex = native.Exec()
        self.ex.stream = ctypes.c_void_p(self.stream.cuda_stream)
        self.L = native.lib()
        self.resident = collections.OrderedDict()   # bid -> _Batch (LRU order)
        self.resident_bytes = 0
        self.results: dict[int, RequestResult] = {}
        self.requests: dict[int, Request] = {}

    # -- memory accounting ---------------------------------------------------
    def _used(self, inflight):
        return self.resident_bytes + sum(b.reserve for b in inflight)

    def _evict_one(self):
        bid, b = self.resident.popitem(last=False)
        self.resident_bytes -= b.bytes
        self.L.pyrb_built_free(ctypes.byref(self.ex), ctypes.byref(b.built))
        for r in b.reqs:
            self.results.pop(r.rid, None)
        return b

    def release_all(self):
        while self.resident:
            self._evict_one()

    # -- one batch -------------------------------------------------------------
    def _launch(self, bid, reqs):
        import torch
        pool = self.pool
        K = len(reqs)
        chunk = np.array([r.chunk for r in reqs], dtype=np.int64)
        log2s = np.ascontiguousarray(pool.log2s[chunk])
        sizes = pool.sizes[chunk].astype(np.uint64)
        voff = np.zeros(K + 1, np.uint32)
        voff[1:] = np.cumsum(sizes).astype(np.uint32)
        starts = np.ascontiguousarray(pool.starts[chunk])
        elens = np.array([len(r.edits) for r in reqs], dtype=np.uint64)
        eoff = np.zeros(K + 1, np.uint32)
        eoff[1:] = np.cumsum(elens).astype(np.uint32)
        edits = np.concatenate([r.edits for r in reqs]) if eoff[-1] else np.zeros((1, 4), np.uint32)
        with torch.cuda.stream(self.stream):
            def up(a):
                t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                return t.to("cuda", non_blocking=True)
            d_log2 = up(log2s.view(np.int32))
            d_voff = up(voff.view(np.int32))
            d_eoff = up(eoff.view(np.int32))
            d_starts = up(starts.view(np.int64))
            d_edits = up(np.ascontiguousarray(edits, dtype=np.uint32).view(np.int32))
        roots = torch.zeros(K, dtype=torch.int32).pin_memory()
        first = torch.zeros(K, dtype=torch.int32).pin_memory()
        fprim = torch.zeros(K, dtype=torch.int32).pin_memory()
        counts = torch.zeros(native.COUNTS_WORDS, dtype=torch.int32).pin_memory()
        keep = [log2s, d_log2, d_voff, d_eoff, d_starts, d_edits]
        bd = native.Batch(count=K, log2_host=log2s.ctypes.data, log2=d_log2.data_ptr(),
                          voxels=pool.voxels.data_ptr(), voxel_offsets=d_voff.data_ptr(),
                          edits=d_edits.data_ptr() if eoff[-1] else 0, edit_offsets=d_eoff.data_ptr() if eoff[-1] else 0,
                          voxel_total=int(voff[-1]), edit_total=int(eoff[-1]), voxel_starts=d_starts.data_ptr())
        built = native.BuiltC()
        native.check(self.L.pyrb_build_batch_async(ctypes.byref(self.ex), ctypes.byref(bd), self.rt,
                                                   roots.data_ptr(), first.data_ptr(), fprim.data_ptr(),
                                                   counts.data_ptr(), ctypes.byref(built)))
        done = torch.cuda.Event(enable_timing=True)
        done.record(self.stream)
        entries = int(voff[-1]) + int(eoff[-1])
        reserve = self.BYTES_PER_ENTRY * entries + self.BYTES_FIXED
        return _Batch(bid, reqs, built, done, keep, roots, first, fprim, counts, entries, reserve)

    def _retire(self, b, t0_event, stats):
        native.check(self.L.pyrb_build_finish(ctypes.c_void_p(b.counts.data_ptr()), ctypes.byref(b.built)))
        st = native.Stats()
        self.L.pyrb_last_stats(ctypes.byref(st))
        b.bytes = int(st.output_bytes)          # scratch is released, the outputs stay resident
        done_ms = t0_event.elapsed_time(b.done)
        roots = b.roots.numpy().view(np.uint32)
        first = b.first.numpy().view(np.uint32)
        fprim = b.fprim.numpy().view(np.uint32)
        for k, r in enumerate(b.reqs):
            lat = done_ms - r.arrival * 1e3
            self.results[r.rid] = RequestResult(b.bid, int(roots[k]), int(first[k]), int(fprim[k]), lat)
            stats.latencies_ms.append(lat)
        stats.voxels += b.built.voxel_count
        b.keep = None
        self.resident[b.bid] = b
        self.resident_bytes += b.bytes

    # -- the serving loop ------------------------------------------------------
    def serve(self, requests: list[Request], realtime: bool = True) -> ServeStats:
        import torch
        stats = ServeStats(requests=len(requests))
        for r in requests:
            self.requests[r.rid] = r
        order = sorted(requests, key=lambda r: r.arrival)
        pending = collections.deque()
        inflight = collections.deque()
        t0_event = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0_event.record(self.stream)
        t0 = time.perf_counter()
        nxt, bid = 0, 0
        while nxt < len(order) or pending or inflight:
            now = (time.perf_counter() - t0) if realtime else float("inf")
            while nxt < len(order) and order[nxt].arrival <= now:
                pending.append(order[nxt])
                nxt += 1
            while inflight and inflight[0].done.query():
                self._retire(inflight.popleft(), t0_event, stats)
            launched = False
            if pending and len(inflight) < self.max_inflight:
                reqs, vox = [], 0
                while pending and (not reqs or vox + int(self.pool.sizes[pending[0].chunk]) <= self.max_batch_voxels):
                    r = pending.popleft()
                    reqs.append(r)
                    vox += int(self.pool.sizes[r.chunk]) + len(r.edits)
                need = self.BYTES_PER_ENTRY * vox + self.BYTES_FIXED
                while self.resident and self._used(inflight) + need > self.budget:
                    self._evict_one()
                    stats.evictions += 1
                if self._used(inflight) + need <= self.budget or not inflight:
                    b = self._launch(bid, reqs)
                    bid += 1
                    inflight.append(b)
                    stats.batches += 1
                    stats.max_batch_requests = max(stats.max_batch_requests, len(reqs))
                    stats.peak_bytes = max(stats.peak_bytes, self._used(inflight))
                    launched = True
                else:
                    for r in reversed(reqs):
                        pending.appendleft(r)
            if not launched and inflight and (not pending or len(inflight) >= self.max_inflight):
                # nothing to launch: wait for the oldest batch (realtime: poll, new requests may arrive)
                if realtime:
                    time.sleep(20e-6)
                else:
                    inflight[0].done.synchronize()
        end = torch.cuda.Event(enable_timing=True)
        end.record(self.stream)
        end.synchronize()
        stats.duration_s = t0_event.elapsed_time(end) / 1e3
        return stats

    # -- access to a served result (tests) -------------------------------------
    def download(self, rid: int):
        """Host copy of the whole batch buffers holding request `rid` plus its result."""
        from .gpu_build import Built
        res = self.results[rid]
        b = self.resident[res.batch]
        torch_stream = self.stream.cuda_stream
        view = Built(b.built, torch_stream)
        host = view.download()
        view._c = None  # the server owns the buffers
        return res, host
