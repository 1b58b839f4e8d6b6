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
* admission is by memory accounting: all scratch (dedup tables, sort buffers) and all
  results are sub-allocated from one fixed device arena of `budget_bytes` (first fit
  with coalescing); a batch is launched only when its estimated need fits into the
  largest free range, evicting the least recently used results first;
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


class RangeArena:
    """First-fit range allocator with coalescing over one fixed device buffer (the
    reference's pool allocator, src/range_alloc.zig:25-58). Ranges freed while a batch
    is being enqueued are held back until that batch has completed on the GPU."""

    ALIGN = 256

    def __init__(self, nbytes: int):
        import torch
        self.size = nbytes // self.ALIGN * self.ALIGN
        self.buf = torch.empty(self.size, dtype=torch.uint8, device="cuda")
        self.base = self.buf.data_ptr()
        self.free = [(0, self.size)]        # sorted (offset, length)
        self.live = {}                      # address -> length
        self.used = 0
        self.peak = 0
        self.defer_to = None                # list collecting deferred frees

    def alloc(self, nbytes: int) -> int:
        n = (max(nbytes, 1) + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        for i, (off, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (off + n, ln - n)
                addr = self.base + off
                self.live[addr] = n
                self.used += n
                self.peak = max(self.peak, self.used)
                return addr
        return 0

    def release(self, addr: int) -> None:
        n = self.live.pop(addr)
        self.used -= n
        off = addr - self.base
        import bisect
        i = bisect.bisect_left(self.free, (off, 0))
        # coalesce with the neighbours
        if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == off:
            i -= 1
            off, n = self.free[i][0], self.free[i][1] + n
            self.free.pop(i)
        if i < len(self.free) and off + n == self.free[i][0]:
            n += self.free[i][1]
            self.free.pop(i)
        self.free.insert(i, (off, n))

    def free_cb(self, addr: int) -> None:
        if self.defer_to is not None:
            self.defer_to.append(addr)
        else:
            self.release(addr)

    def largest_free(self) -> int:
        return max((ln for _, ln in self.free), default=0)


class _Slot:
    """Preallocated pinned staging and device buffers of one in-flight batch."""

    def __init__(self, max_chunks, max_edits):
        import torch
        K, E = max_chunks, max_edits

        def pin(n, dt):
            return torch.zeros(n, dtype=dt).pin_memory()

        def dev(n, dt):
            return torch.zeros(n, dtype=dt, device="cuda")

        self.h_log2, self.d_log2 = pin(K, torch.int32), dev(K, torch.int32)
        self.h_voff, self.d_voff = pin(K + 1, torch.int32), dev(K + 1, torch.int32)
        self.h_eoff, self.d_eoff = pin(K + 1, torch.int32), dev(K + 1, torch.int32)
        self.h_starts, self.d_starts = pin(K, torch.int64), dev(K, torch.int64)
        self.h_edits, self.d_edits = pin(4 * max(E, 1), torch.int32), dev(4 * max(E, 1), torch.int32)
        self.roots, self.first, self.fprim = pin(K, torch.int32), pin(K, torch.int32), pin(K, torch.int32)
        self.counts = pin(native.COUNTS_WORDS, torch.int32)
        self.log2_np = np.zeros(K, np.uint32)


class _Batch:
    def __init__(self, bid, reqs, built, done, slot, entries, reserve, deferred):
        self.bid, self.reqs, self.built, self.done, self.slot = bid, reqs, built, done, slot
        self.entries, self.reserve, self.bytes = entries, reserve, reserve
        self.deferred = deferred   # scratch ranges to release once the batch is done


class ChunkServer:
    # scratch + output bound per entry of a batch build (sort buffers, unique keys and
    # attributes, bricks, dedup tables, node bound), a safe over-estimate
    BYTES_PER_ENTRY = 96
    BYTES_FIXED = 4 << 20

    def __init__(self, pool: ChunkPool, budget_bytes: int = 40 << 30, max_batch_voxels: int = 128 << 20,
                 max_inflight: int = 2, rt_log2: int = 5, stream=None, max_batch_requests: int = 1024,
                 max_edits_per_request: int = 64):
        import torch
        self.pool = pool
        self.max_batch_requests = max_batch_requests
        self.max_edits = max_edits_per_request
        self.free_slots = [_Slot(max_batch_requests, max_batch_requests * max_edits_per_request)
                           for _ in range(max_inflight)]
        # all scratch (dedup tables, sort buffers) and every result live in one fixed arena
        self.arena = RangeArena(budget_bytes)
        self._alloc_cb = native.ALLOC_FN(lambda ctx, n: self._alloc(n))
        self._free_cb = native.FREE_FN(lambda ctx, a: self.arena.free_cb(a))
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
        self.keep_results = True
        self.ex.alloc = self._alloc_cb
        self.ex.free = self._free_cb
        self._evictions = 0

    def _alloc(self, nbytes: int) -> int:
        a = self.arena.alloc(nbytes)
        while not a and self.resident:      # make room: evict least recently used results
            self._evict_one()
            self._evictions += 1
            a = self.arena.alloc(nbytes)
        return a

    # -- memory accounting ---------------------------------------------------
    def _used(self, inflight):
        return self.arena.used

    def _evict_one(self):
        bid, b = self.resident.popitem(last=False)
        self.resident_bytes -= b.bytes
        saved, self.arena.defer_to = self.arena.defer_to, None   # a finished batch: release at once
        try:
            self.L.pyrb_built_free(ctypes.byref(self.ex), ctypes.byref(b.built))
        finally:
            self.arena.defer_to = saved
        for r in b.reqs:
            self.results.pop(r.rid, None)
        return b

    def release_all(self):
        while self.resident:
            self._evict_one()

    # -- one batch -------------------------------------------------------------
    def _launch(self, bid, reqs):
        pool = self.pool
        slot = self.free_slots.pop()
        K = len(reqs)
        chunk = np.fromiter((r.chunk for r in reqs), dtype=np.int64, count=K)
        log2s = slot.log2_np[:K]
        log2s[:] = pool.log2s[chunk]
        voff = slot.h_voff.numpy()[:K + 1].view(np.uint32)
        voff[0] = 0
        np.cumsum(pool.sizes[chunk], out=voff[1:])
        slot.h_log2.numpy()[:K] = log2s.view(np.int32)
        slot.h_starts.numpy()[:K] = pool.starts[chunk].view(np.int64)
        eoff = slot.h_eoff.numpy()[:K + 1].view(np.uint32)
        eoff[0] = 0
        np.cumsum(np.fromiter((len(r.edits) for r in reqs), dtype=np.uint32, count=K), out=eoff[1:])
        ne = int(eoff[K])
        if ne:
            he = slot.h_edits.numpy()[:4 * ne].reshape(ne, 4).view(np.uint32)
            o = 0
            for r in reqs:
                m = len(r.edits)
                if m:
                    he[o:o + m] = r.edits
                    o += m
        import torch
        with torch.cuda.stream(self.stream):
            slot.d_log2[:K].copy_(slot.h_log2[:K], non_blocking=True)
            slot.d_voff[:K + 1].copy_(slot.h_voff[:K + 1], non_blocking=True)
            slot.d_eoff[:K + 1].copy_(slot.h_eoff[:K + 1], non_blocking=True)
            slot.d_starts[:K].copy_(slot.h_starts[:K], non_blocking=True)
            if ne:
                slot.d_edits[:4 * ne].copy_(slot.h_edits[:4 * ne], non_blocking=True)
        bd = native.Batch(count=K, log2_host=log2s.ctypes.data, log2=slot.d_log2.data_ptr(),
                          voxels=pool.voxels.data_ptr(), voxel_offsets=slot.d_voff.data_ptr(),
                          edits=slot.d_edits.data_ptr() if ne else 0, edit_offsets=slot.d_eoff.data_ptr() if ne else 0,
                          voxel_total=int(voff[K]), edit_total=ne, voxel_starts=slot.d_starts.data_ptr())
        built = native.BuiltC()
        deferred = []
        self.arena.defer_to = deferred
        try:
            rc = self.L.pyrb_build_batch_async(ctypes.byref(self.ex), ctypes.byref(bd), self.rt,
                                               slot.roots.data_ptr(), slot.first.data_ptr(),
                                               slot.fprim.data_ptr(), slot.counts.data_ptr(), ctypes.byref(built))
        finally:
            self.arena.defer_to = None
        if rc != native.PYRB_OK:
            self.free_slots.append(slot)
            for a in deferred:       # nothing was enqueued that uses them
                self.arena.release(a)
            if rc == native.PYRB_ERROR_OUT_OF_MEMORY:
                return None
            native.check(rc)
        done = torch.cuda.Event(enable_timing=True)
        done.record(self.stream)
        entries = int(voff[K]) + ne
        reserve = self.BYTES_PER_ENTRY * entries + self.BYTES_FIXED
        return _Batch(bid, reqs, built, done, slot, entries, reserve, deferred)

    def _retire(self, b, t0_event, stats):
        slot = b.slot
        native.check(self.L.pyrb_build_finish(ctypes.c_void_p(slot.counts.data_ptr()), ctypes.byref(b.built)))
        st = native.Stats()
        self.L.pyrb_last_stats(ctypes.byref(st))
        b.bytes = int(st.output_bytes)          # scratch is released, the outputs stay resident
        done_ms = t0_event.elapsed_time(b.done)
        K = len(b.reqs)
        roots = slot.roots.numpy()[:K].view(np.uint32).copy()
        first = slot.first.numpy()[:K].view(np.uint32).copy()
        fprim = slot.fprim.numpy()[:K].view(np.uint32).copy()
        arrivals = np.fromiter((r.arrival for r in b.reqs), dtype=np.float64, count=K)
        lats = done_ms - arrivals * 1e3
        stats.latencies_ms.extend(lats.tolist())
        if self.keep_results:
            for k, r in enumerate(b.reqs):
                self.results[r.rid] = RequestResult(b.bid, int(roots[k]), int(first[k]), int(fprim[k]), float(lats[k]))
        stats.voxels += b.built.voxel_count
        self.free_slots.append(slot)
        b.slot = None
        for a in b.deferred:
            self.arena.release(a)
        b.deferred = []
        self.resident[b.bid] = b
        self.resident_bytes += b.bytes

    # -- the serving loop ------------------------------------------------------
    def serve(self, requests: list[Request], realtime: bool = True) -> ServeStats:
        import torch
        stats = ServeStats(requests=len(requests))
        too_many = [r.rid for r in requests if len(r.edits) > self.max_edits]
        if too_many:
            raise ValueError(f"requests {too_many[:4]} carry more than {self.max_edits} edits")
        if self.keep_results:
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
                while pending and len(reqs) < self.max_batch_requests and (
                        not reqs or vox + int(self.pool.sizes[pending[0].chunk]) <= self.max_batch_voxels):
                    r = pending.popleft()
                    reqs.append(r)
                    vox += int(self.pool.sizes[r.chunk]) + len(r.edits)
                need = self.BYTES_PER_ENTRY * vox + self.BYTES_FIXED
                while self.resident and self.arena.largest_free() < need:
                    self._evict_one()
                    stats.evictions += 1
                b = self._launch(bid, reqs) if (self.arena.largest_free() >= need or not inflight) else None
                if b is not None:
                    bid += 1
                    inflight.append(b)
                    stats.batches += 1
                    stats.max_batch_requests = max(stats.max_batch_requests, len(reqs))
                    stats.peak_bytes = max(stats.peak_bytes, self.arena.peak)
                    launched = True
                else:
                    if not inflight:
                        raise RuntimeError(f"a batch of {vox} voxels does not fit into the {self.budget}-byte arena")
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
        stats.evictions += self._evictions
        self._evictions = 0
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
