#!/usr/bin/env python
"""Benchmark of the B200 DAG build (one JSON line on rank 0).

Workload (N=1 and every rank of N>1): plain single-chunk build of a 256^3 grid of
thresholded 3-octave value noise (~30% solid, materials 1..8 per 8^3 block) with a
0.5% set/remove edit overlay applied in the same build -- seeded synthetic input of
the shapes the metric is quoted on. A step is one full build (encode, onesweep
sort, unique, bricks/leaves, all node levels, prims) of that input.

  value   unique voxels built per second over all ranks, device time of the build
          with the input resident in HBM (CUDA events per step; L2 is flushed by a
          512 MiB write between steps, outside the timed events).
  e2e     the same metric through the public C ABI with HOST input, wall clock: a
          stream of builds (pyrb_build_async) where every step uploads its own
          PyrVoxel input from pinned memory on a copy stream and reads its counts
          back; uploads overlap the previous build. The one-call-at-a-time figure
          (pyrb_geometry_build + PYRB_BUILD_HOST_INPUT) is reported beside it.
  roofline  the dominant HBM kernel of the build (largest share of its per-stage CUDA
          event time): algorithmic bytes per launch / mean launch time, against the
          measured HBM copy bandwidth; "kernels" lists every HBM kernel the same way
          (byte formulas in kernel_roofline).
  cpu_baseline  the reference's CPU builder (restated in oracle/: hash-map overlay
          merge + buildPoints, src/dag_builder.zig) on one host core, one build.

--impl reference runs that CPU builder alone (rank 0) on the same workload.
Multi-GPU: every rank builds its own copy (replicas; a single volume does not
shard), value = sum over ranks, time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DAG-build voxels/s"
WORKLOAD = "plain single-chunk build: 256^3 3-octave value noise > 70th percentile (~30% solid), +0.5% set/remove edits"


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


WORKLOAD_BERNOULLI = ("worst-case dedup single build: 1024^3 i.i.d. Bernoulli(0.15) occupancy, material "
                      "uniform 1..255, +10^6 uniform set/remove edits")
# name -> (edge log2, rt_log2, description, CPU-baseline sample octant log2 or None for the whole grid)
SPECS = {
    "noise256": (8, 7, WORKLOAD, None),
    "bernoulli1024": (10, 7, WORKLOAD_BERNOULLI, 8),
    # the same generator at edge 512 (2^17 edits): a case small enough for ncu captures
    "bernoulli512": (9, 7, WORKLOAD_BERNOULLI.replace("1024^3", "512^3").replace("10^6", "2^17"), 8),
}


def make_input(name="noise256"):
    from pyrit_b200 import workloads as wl
    if name == "bernoulli1024":
        vox = wl.bernoulli_grid(10, 0)
        ed = wl.uniform_edits(10, 1_000_000, 0)
    elif name == "bernoulli512":
        vox = wl.bernoulli_grid(9, 0)
        ed = wl.uniform_edits(9, 1 << 17, 0)
    else:
        vox = wl.noise_grid(8, 0)
        ed = wl.noise_edits(8, 0)
    return vox, ed, np.concatenate([vox, ed])


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of `kernel` on `workload` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.strip().strip("|").split("|")
        if len(parts) >= 3 and parts[0].strip() == kernel and parts[1].strip().startswith(workload + ":"):
            try:
                return int(parts[2].strip())
            except ValueError:
                return None
    return None


class ClockSampler:
    """NVML samples of SM clock and clock-event reasons while the timed region runs."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device_index: int):
        self.samples, self.reasons, self.ok = [], 0, False
        self._stop = threading.Event()
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            try:
                self.h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None

    def _reasons(self):
        try:
            return self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except Exception:
            return self.nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= int(self._reasons())
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        names = [n for b, n in self.REASONS.items() if self.reasons & b and b != 0x1]
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples)}


def cpu_builder_time(vox, ed, reps=1, log2=8):
    """Reference CPU builder (oracle restatement) on one core: seconds per build, voxels."""
    from oracle import oracle as orc
    best, n = None, 0
    for _ in range(reps):
        t = time.perf_counter()
        d = orc.cpu_build_overlay(log2, vox, ed)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
        n = d.voxel_count
    return best, n


def stage_profile(log2, rt, dpts, sptr, flush, steps):
    """Mean duration (ms) of every stage of a build: CUDA events after every launch
    (pyrb_profile_enable), over `steps` builds with L2 flushed before each."""
    from pyrit_b200 import gpu_build, native
    L = native.lib()
    L.pyrb_profile_enable(1)
    stage = {}
    try:
        for s in range(steps):
            flush.fill_(s & 0xFF)
            b = gpu_build.build(log2, rt, dpts, stream=sptr)
            ms = (ctypes.c_float * 256)()
            names = ctypes.create_string_buffer(256 * 32)
            k = L.pyrb_profile_read(ms, names, 32, 256)
            for i in range(min(k, 256)):
                nm = names.raw[i * 32:(i + 1) * 32].split(b"\0")[0].decode()
                stage.setdefault(nm, []).append(ms[i])
            b.free()
    finally:
        L.pyrb_profile_enable(0)
    return {k: statistics.mean(v) for k, v in stage.items()}


def path_name(stage_ms):
    """How the build ordered its voxels, from its stages."""
    if "bucket_count" in stage_ms:
        return "brick buckets"
    return "cell grid" if "grid_scatter" in stage_ms else "sort"


def kernel_roofline(stage_ms, st, n_in, n_u, leaves, key_bytes, peak, cells=0):
    """Algorithmic bytes / CUDA-event time of the build's HBM kernels against `peak`
    (GB/s). Bytes per launch (the roofline basis of the design notes):
      grid_scatter  n_in (16 + 8)                read PyrVoxels, one 8-byte cell update each
      grid_count    8 cells                      read every cell (its 32-byte sector holds 4)
      grid_write    8 cells + 12 n_u + 20 B      read every cell, write keys, attributes, bricks
      bucket_count  n_in (16 + 4)                read PyrVoxels, add to the brick's counter
      bucket_scatter n_in (16 + 4 + 9)           read PyrVoxels, take a slot, write the 9-byte record
      bucket_tile_count  9 n_in + 4 nb           read the records and the bucket bounds (nb bricks)
      bucket_tile_write  9 n_in + 4 nb + 12 n_u + 20 B
      encode_hist   n_in (16 + kb + 4)           read PyrVoxels, write key + value
      sort_pass     n_in 2 (kb + 4)              read and write key + value
      unique_brick  n_in (kb + 4) + 12 n_u + 20 B
      leaf_part     20 B; leaf_insert 28 B; leaf_own 16 B + 8 L
      node level l  20 C + 28 P + 4 W            children C, parents P, words W written
    with B bricks, L leaves, W = 2 U + C U / P for U unique parents. Each entry also
    carries "share": its part of the build's summed stage time (a sort pass: all passes)."""
    B = int(st.brick_count)
    out = {}
    total_ms = sum(stage_ms.values()) or 1.0

    def add(name, ms, nbytes, launches=1):
        if ms and ms > 0:
            gbs = nbytes / (ms / 1e3) / 1e9
            out[name] = {"ms": round(ms, 4), "alg_bytes": int(nbytes), "gbs": round(gbs, 1),
                         "frac": round(gbs / peak, 4), "share": round(launches * ms / total_ms, 4)}

    add("grid_scatter", stage_ms.get("grid_scatter"), n_in * 24)
    add("grid_count", stage_ms.get("grid_count"), 8 * cells)
    add("grid_write", stage_ms.get("grid_write"), 8 * cells + 12 * n_u + 20 * B)
    nb = cells // 64
    add("bucket_count", stage_ms.get("bucket_count"), n_in * 20)
    add("bucket_scatter", stage_ms.get("bucket_scatter"), n_in * 29)
    add("bucket_tile_count", stage_ms.get("bucket_tile_count"), 9 * n_in + 4 * nb)
    add("bucket_tile_write", stage_ms.get("bucket_tile_write"), 9 * n_in + 4 * nb + 12 * n_u + 20 * B)
    add("encode_hist", stage_ms.get("encode_hist"), n_in * (16 + key_bytes + 4))
    sort_keys = [k for k in stage_ms if k.startswith("sort_pass")]
    if sort_keys:
        add("sort_pass", statistics.mean(stage_ms[k] for k in sort_keys), n_in * 2 * (key_bytes + 4), len(sort_keys))
    add("unique_brick", stage_ms.get("unique_brick"), n_in * (key_bytes + 4) + 12 * n_u + 20 * B)
    add("leaf_part", stage_ms.get("leaf_part"), 20 * B)
    add("leaf_insert", stage_ms.get("leaf_insert"), 28 * B)
    add("leaf_own", stage_ms.get("leaf_own"), 16 * B + 8 * leaves)
    def node_bytes(lv):
        C = B if lv == 2 else int(st.level_parents[lv - 1])
        P, U = int(st.level_parents[lv]), int(st.level_unique[lv])
        W = 2 * U + (C * U // P if P else 0)
        return 20 * C + 28 * P + 4 * W

    for lv in range(2, 24):
        nb, no = stage_ms.get("node_build:%d" % lv), stage_ms.get("node_own:%d" % lv)
        if nb is None or no is None:
            continue
        add("node_dedup:%d" % lv, nb + no, node_bytes(lv))
    return out


def sub_volume(pts, log2):
    """Entries of the workload inside the octant [0, 2^log2)^3 (a bounded CPU sample)."""
    m = (pts[:, 0] < (1 << log2)) & (pts[:, 1] < (1 << log2)) & (pts[:, 2] < (1 << log2))
    return pts[m]


def run_reference(args):
    rank = _env_int("RANK", 0)
    if rank != 0:
        return 0
    full, _, desc, _ = SPECS[args.workload]
    vox, ed, _ = make_input(args.workload)
    # one full 256^3 build takes ~1-3 s on one core: shrink the per-step sample for long runs
    runs = args.steps + args.warmup
    log2 = 8 if runs <= 50 else (7 if runs <= 400 else 6)
    log2 = min(log2, full)
    if log2 < full:
        vox, ed = sub_volume(vox, log2), sub_volume(ed, log2)
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as orc

    # The reference builder is single-threaded; the host's cores each build their own
    # copy of the sample at once (ctypes releases the GIL), the way independent chunk
    # builds spread over a CPU.
    threads = max(1, min(os.cpu_count() or 1, 32))
    pool = ThreadPoolExecutor(threads)

    def build_one(_):
        return orc.cpu_build_overlay(log2, vox, ed).voxel_count

    def one():
        t = time.perf_counter()
        counts = list(pool.map(build_one, range(threads)))
        return time.perf_counter() - t, counts[0]

    for _ in range(args.warmup):
        one()
    times, n = [], 0
    for _ in range(args.steps):
        dt, n = one()
        times.append(dt)
    pool.shutdown()
    total = sum(times)
    value = threads * n * len(times) / total
    sample = ("per step %d concurrent builds of the whole workload" % threads if log2 == full else
              "per step %d concurrent builds of the %d^3 octant of the workload (same voxels and edits inside it)"
              % (threads, 1 << log2))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": desc, "log2_size": full, "sample_log2": log2, "unique_voxels_per_sample": n},
        "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": threads, "kind": "port",
                         "sample": sample + ": hash-map edit merge + buildPoints "
                                   "(src/dag_builder.zig restated in oracle/dag_cpu.cpp), one build per thread"},
        "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    from pyrit_b200 import gpu_build, native

    rank, world, local = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1), _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    L = native.lib()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    LOG2, RT, desc, cpu_sample_log2 = SPECS[args.workload]
    vox, ed, pts = make_input(args.workload)
    n_in = len(pts)
    dpts = torch.from_numpy(pts.view(np.int32)).cuda()
    host = torch.from_numpy(pts.view(np.int32)).pin_memory()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(native.COUNTS_WORDS, dtype=torch.int32).pin_memory()
    counts_ptr = counts.data_ptr()
    ex = native.Exec()
    ex.stream = ctypes.c_void_p(sptr)

    def build_async():
        out = native.BuiltC()
        native.check(L.pyrb_build_async(ctypes.byref(ex), LOG2, RT, 0, 0, 0, dpts.data_ptr(), n_in,
                                        ctypes.c_void_p(counts_ptr), ctypes.byref(out)))
        return out

    def release(out):
        L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(out))

    # warm-up (also validates one result against itself between runs)
    for _ in range(max(args.warmup, 1)):
        o = build_async()
        release(o)
    stream.synchronize()
    o = native.BuiltC()
    native.check(L.pyrb_build_finish(ctypes.c_void_p(counts_ptr), ctypes.byref(o)))
    n_u = o.voxel_count
    st = gpu_build.last_stats()
    launches_per_build = st.kernel_launches

    # timed region: K builds, L2 flushed between them outside the events
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            flush.fill_(s & 0xFF)
            evs[s][0].record(stream)
            o = build_async()
            evs[s][1].record(stream)
            release(o)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    o = native.BuiltC()
    native.check(L.pyrb_build_finish(ctypes.c_void_p(counts_ptr), ctypes.byref(o)))
    assert o.voxel_count == n_u, "result changed between runs"
    sizes = {"leaves": o.leaf_count, "node_words": o.node_words, "prims": o.prim_count}
    step_ms = [a.elapsed_time(b) for a, b in evs]
    t_ms = sum(step_ms)
    t_max = torch.tensor([t_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    t_ms = float(t_max.item())
    value = world * n_u * args.steps / (t_ms / 1e3)

    # per-stage profile (CUDA events after every launch of the build)
    stage_ms = stage_profile(LOG2, RT, dpts, sptr, flush, min(args.steps, 20))
    key_bytes = 4 if 3 * LOG2 + 1 <= 32 else 8
    peak, peak_kind = load_peaks()
    # the dominant kernel: the largest share of the build's stage time (a per-level
    # node dedup is a pair of kernels, listed in "kernels" but not a candidate)
    kernels = kernel_roofline(stage_ms, st, n_in, n_u, sizes["leaves"], key_bytes, peak,
                              cells=(1 << (3 * LOG2)) if st.sort_passes == 0 else 0)
    names = {"grid_scatter": "k_grid_scatter", "grid_count": "k_grid_count", "grid_write": "k_grid_write",
             "sort_pass": "k_sort_pass", "encode_hist": "k_encode_hist", "unique_brick": "k_unique",
             "leaf_insert": "k_leaf_insert", "leaf_own": "k_leaf_own", "bucket_count": "k_bkt_count",
             "bucket_scatter": "k_bkt_scatter", "bucket_tile_count": "k_grid_count<bucket>",
             "bucket_tile_write": "k_grid_write<bucket>"}
    dom = max((k for k in kernels if k in names), key=lambda k: kernels[k]["share"])
    dom_kernel = names[dom]
    dom_bytes, dom_ms = kernels[dom]["alg_bytes"], kernels[dom]["ms"]
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = committed_traffic(dom_kernel, args.workload)

    # whole-build algorithmic bytes (read input once; write keys+attrs, leaves, nodes, prims)
    alg_bytes = 16 * n_in + 12 * n_u + 8 * sizes["leaves"] + 4 * sizes["node_words"] + 40 * sizes["prims"]
    hbm_gbs = alg_bytes * args.steps / (t_ms / 1e3) / 1e9 / world

    # e2e through the public C ABI with host input
    e2e_steps = min(args.steps, 20)
    e2e_times = []
    if dist:
        dist.barrier()
    for s in range(e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b = gpu_build.geometry_build(LOG2, RT, host.numpy().view(np.uint32), stream=sptr)
        e2e_times.append(time.perf_counter() - t0)
        assert b.voxel_count == n_u
        b.free()
    e2e_s = torch.tensor([sum(e2e_times)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
    e2e_sync_value = world * n_u * e2e_steps / float(e2e_s.item())

    # e2e of a stream of builds through the public asynchronous API: every step uploads
    # its own input from pinned host memory (on a copy stream) and reads its counts back
    # (pyrb_build_async -> pinned counts, pyrb_build_finish); the upload of step k+1
    # overlaps the build of step k (two device input buffers).
    cstream = torch.cuda.Stream()
    dbuf = [torch.empty_like(dpts), torch.empty_like(dpts)]
    pinned_counts = [torch.zeros(native.COUNTS_WORDS, dtype=torch.int32).pin_memory() for _ in range(e2e_steps)]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    built = [torch.cuda.Event(), torch.cuda.Event()]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        k = s & 1
        with torch.cuda.stream(cstream):
            if s >= 2:
                cstream.wait_event(built[k])
            dbuf[k].copy_(host, non_blocking=True)
            copied[k].record(cstream)
        stream.wait_event(copied[k])
        o = native.BuiltC()
        native.check(L.pyrb_build_async(ctypes.byref(ex), LOG2, RT, 0, 0, 0, dbuf[k].data_ptr(), n_in,
                                        ctypes.c_void_p(pinned_counts[s].data_ptr()), ctypes.byref(o)))
        built[k].record(stream)
        release(o)
    torch.cuda.synchronize()
    t_pipe = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    for s in range(e2e_steps):
        f = native.BuiltC()
        native.check(L.pyrb_build_finish(ctypes.c_void_p(pinned_counts[s].data_ptr()), ctypes.byref(f)))
        assert f.voxel_count == n_u, "pipelined build changed the result"
    if dist:
        dist.all_reduce(t_pipe, op=dist.ReduceOp.MAX)
    e2e_value = world * n_u * e2e_steps / float(t_pipe.item())
    del dbuf

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        if cpu_sample_log2 is None:
            dt, n = cpu_builder_time(vox, ed, reps=1, log2=LOG2)
            what = "one full build of the same workload"
        else:
            dt, n = cpu_builder_time(sub_volume(vox, cpu_sample_log2), sub_volume(ed, cpu_sample_log2), reps=1,
                                     log2=cpu_sample_log2)
            what = "one build of the %d^3 octant of the same workload (its voxels and edits)" % (1 << cpu_sample_log2)
        cpu = {"value": n / dt, "unit": "voxels/s", "cores": 1, "kind": "port",
               "sample": what + ": hash-map edit merge + buildPoints "
                         "(src/dag_builder.zig restated in oracle/dag_cpu.cpp), single thread, %.2f s" % dt}

    # dedup ratio per node level: parents formed / unique nodes kept (level 2 = nodes over bricks)
    dedup = {str(lv): {"parents": int(st.level_parents[lv]), "unique": int(st.level_unique[lv]),
                       "ratio": (st.level_parents[lv] / st.level_unique[lv]) if st.level_unique[lv] else None}
             for lv in range(2, LOG2)}

    # the other configurations of the metric, on one GPU: the batched build of 1024
    # mixed chunks against the per-chunk loop, served requests at 20k/s, and the
    # worst-case 1024^3 build with its per-kernel roofline
    extras = {}
    if world == 1 and not args.no_extras:
        for name, fn in (("batched", lambda: run_batched(args, emit=False)),
                         ("served", lambda: run_served(args, emit=False)),
                         ("worst_case", lambda: run_worst_case(args))):
            try:
                extras[name] = fn()
            except Exception as exc:  # reported in the line, the headline stands
                extras[name] = {"error": "%s: %s" % (type(exc).__name__, exc)}
            gpu_build.set_tuning(0, 0, 50)  # the autotuned setting of one form does not leak into the next
            torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded value noise + edit overlay)",
            "config": {"workload": desc, "log2_size": LOG2, "rt_log2": RT, "entries": n_in, "unique_voxels": n_u,
                       "bricks": st.brick_count, "leaves": sizes["leaves"], "node_words": sizes["node_words"],
                       "prims": sizes["prims"], "sort_passes": st.sort_passes, "radix_bits": st.radix_bits,
                       "l2": "flushed between steps (512 MiB write outside the timed events)",
                       "key_bits": 8 * key_bytes, "path": path_name(stage_ms),
                       "dedup_per_level": dedup,
                       "scratch_bytes": int(st.scratch_bytes), "output_bytes_bound": int(st.output_bytes),
                       "parallelism": "replicas" if world > 1 else "single"},
            "hbm_gbs": hbm_gbs,
            "roofline": {"bound": "hbm", "kernel": dom_kernel, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": dom_bytes, "mean_launch_ms": dom_ms,
                         "share_of_build": kernels[dom]["share"]},
            "kernels": kernels,
            "stages_ms": {k: round(v, 4) for k, v in stage_ms.items()},
            "e2e": {"value": e2e_value, "unit": "voxels/s", "h2d_bytes_per_step": 16 * n_in,
                    "d2h_bytes_per_step": 4 * native.COUNTS_WORDS,
                    "ms_per_step": 1e3 * float(t_pipe.item()) / e2e_steps,
                    "how": "pyrb_build_async per step on an uploaded copy of its PyrVoxel input (pinned host, copy "
                           "stream, double-buffered) + counts read back; uploads overlap the previous build",
                    "sync_single_call": {"value": e2e_sync_value,
                                         "ms_per_step": 1e3 * float(e2e_s.item()) / e2e_steps,
                                         "how": "pyrb_geometry_build with PYRB_BUILD_HOST_INPUT, one call at a time"}},
            "gpu_launches": launches_per_build * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_worst_case(args, reps=3):
    """Worst-case dedup build at full size: 1024^3 i.i.d. Bernoulli(0.15) occupancy,
    materials 1..255, +10^6 uniform set/remove edits (162 M entries, 2.6 GB of input in
    HBM). Device time per build (CUDA events, L2 flushed between builds), the
    algorithmic-bytes roofline of every HBM kernel from per-stage events, and the
    dedup ratio (parents formed / unique nodes kept) per level."""
    import torch
    from pyrit_b200 import gpu_build, native
    L = native.lib()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    LOG2, RT, desc, _ = SPECS["bernoulli1024"]
    vox, ed, pts = make_input("bernoulli1024")
    n_in = len(pts)
    dpts = torch.from_numpy(pts.view(np.int32)).cuda()
    del vox, ed, pts
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    counts = torch.zeros(native.COUNTS_WORDS, dtype=torch.int32).pin_memory()
    ex = native.Exec()
    ex.stream = ctypes.c_void_p(sptr)

    def build_async():
        out = native.BuiltC()
        native.check(L.pyrb_build_async(ctypes.byref(ex), LOG2, RT, 0, 0, 0, dpts.data_ptr(), n_in,
                                        ctypes.c_void_p(counts.data_ptr()), ctypes.byref(out)))
        return out

    for _ in range(2):
        L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(build_async()))
    torch.cuda.synchronize()
    times = []
    for s in range(reps):
        flush.fill_(s & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        o = build_async()
        b.record(stream)
        L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(o))
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    o = native.BuiltC()
    native.check(L.pyrb_build_finish(ctypes.c_void_p(counts.data_ptr()), ctypes.byref(o)))
    n_u, leaves = o.voxel_count, o.leaf_count
    st = gpu_build.last_stats()
    stage_ms = stage_profile(LOG2, RT, dpts, sptr, flush, reps)
    # both ways of ordering the voxels, forced (the automatic choice is timed above)
    paths = {}
    old = gpu_build.get_tuning()
    try:
        for name, code in (("sort", native.PATH_SORT), ("grid", native.PATH_GRID), ("bucket", native.PATH_BUCKET)):
            gpu_build.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, code)
            L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(build_async()))
            tt = []
            for s in range(reps):
                flush.fill_(s & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                q = build_async()
                b.record(stream)
                L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(q))
                torch.cuda.synchronize()
                tt.append(a.elapsed_time(b))
            paths[name] = {"ms_per_build": statistics.median(tt),
                           "stages_ms": {k: round(v, 4) for k, v in
                                         stage_profile(LOG2, RT, dpts, sptr, flush, 1).items()}}
    finally:
        gpu_build.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    peak, peak_kind = load_peaks()
    key_bytes = 4 if 3 * LOG2 + 1 <= 32 else 8
    kernels = kernel_roofline(stage_ms, st, n_in, n_u, leaves, key_bytes, peak,
                              cells=(1 << (3 * LOG2)) if st.sort_passes == 0 else 0)
    dedup = {str(lv): {"parents": int(st.level_parents[lv]), "unique": int(st.level_unique[lv]),
                       "ratio": (st.level_parents[lv] / st.level_unique[lv]) if st.level_unique[lv] else None}
             for lv in range(2, LOG2)}
    t = statistics.median(times)
    del dpts, flush
    torch.cuda.empty_cache()
    return {"workload": desc, "entries": n_in, "unique_voxels": n_u, "bricks": int(st.brick_count),
            "leaves": leaves, "ms_per_build": t, "voxels_per_s": n_u / (t / 1e3),
            "sort_passes": int(st.sort_passes), "radix_bits": int(st.radix_bits),
            "peak_gbs": peak, "peak_kind": peak_kind, "kernels": kernels, "dedup_per_level": dedup,
            "path": path_name(stage_ms), "paths_forced": paths,
            "scratch_plus_output_bytes_per_entry": (st.scratch_bytes + st.output_bytes) / n_in,
            "how": "pyrb_build_async on the resident input, CUDA events around each build (median of %d), "
                   "per-stage events from pyrb_profile_enable" % reps}


def path_edit_bench(out, roots, first_voxel, first_prim, log2s, nz, per_chunk=32, reps=3):
    """Path edits over a built batch: `per_chunk` random set/remove edits in every non-empty
    chunk (one job each), through pyrb_path_edit on pools with an arena above the batch.
    Times the call (edit ordering on the host, upload, the three kernels, read-back)."""
    import torch
    from pyrit_b200 import _cudart, gpu_build, native
    rng = np.random.default_rng(5)
    nz = list(nz)
    counts = np.diff(np.concatenate([first_voxel[nz], [out.voxel_count]]).astype(np.int64))
    nxt = np.concatenate([first_prim[nz][1:], [out.prim_count]]).astype(np.int64)
    pcount = nxt - first_prim[nz].astype(np.int64)
    caps = [per_chunk * ((int(log2s[c]) - 2) * 10 + 4) + 8 for c in nz]
    nodes = torch.empty(out.node_words + sum(caps), dtype=torch.int32, device="cuda")
    leaves = torch.empty(out.leaf_count + per_chunk * len(nz), dtype=torch.int64, device="cuda")
    attrs = torch.empty(out.voxel_count + int(counts.sum()) + per_chunk * len(nz), dtype=torch.int32, device="cuda")
    _cudart.dtod(nodes.data_ptr(), out.nodes, 4 * out.node_words)
    _cudart.dtod(leaves.data_ptr(), out.leaves, 8 * out.leaf_count)
    _cudart.dtod(attrs.data_ptr(), out.attrs, 4 * out.voxel_count)
    edits = []
    jobs0 = []
    npos, lpos, apos = out.node_words, out.leaf_count, out.voxel_count
    for k, c in enumerate(nz):
        edge = 1 << int(log2s[c])
        e = np.empty((per_chunk, 4), np.uint32)
        e[:, :3] = rng.integers(0, edge, (per_chunk, 3))
        e[:, 3] = np.where(rng.random(per_chunk) < 0.5, 0, rng.integers(1, 9, per_chunk))
        j = native.PathEditJob(root=int(roots[c]), log2_size=int(log2s[c]), attr_src=int(first_voxel[c]),
                               attr_count=int(counts[k]), attr_a=apos, attr_cap=int(counts[k]) + per_chunk,
                               node_arena=npos, node_cap=caps[k], leaf_arena=lpos, leaf_cap=per_chunk,
                               edit_first=len(edits), edit_count=per_chunk, rt_log2=5,
                               prims=out.prims + 16 * int(first_prim[c]) if pcount[k] else 0,
                               prim_count=int(pcount[k]),
                               aabbs=out.aabbs + 24 * int(first_prim[c]) if pcount[k] else 0, aabbs_keep=1)
        jobs0.append(j)
        edits.extend(e.tolist())
        npos += caps[k]
        lpos += per_chunk
        apos += int(counts[k]) + per_chunk
    edits = np.array(edits, np.uint32)
    times, flags = [], None
    for _ in range(reps):
        jobs = [native.PathEditJob.from_buffer_copy(j) for j in jobs0]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gpu_build.path_edit(nodes, leaves, attrs, jobs, edits)
        times.append(time.perf_counter() - t0)
        flags = np.array([j.out_flags for j in jobs], np.uint32)
    t = min(times)
    return {"jobs": len(nz), "edits": int(len(edits)), "attributes_rewritten": int(counts.sum()),
            "ms": 1e3 * t, "edits_per_s": len(edits) / t,
            "jobs_rebuild_needed": int(((flags & 0x7) != 0).sum()),
            "how": "pyrb_path_edit over every chunk of the batch, %d random set/remove edits each" % per_chunk}


def run_batched(args, emit=True):
    """1024 chunks of the mix (edges 32/64/128/256 with p .4/.3/.2/.1, heightfield tiled per
    chunk and scaled to the edge, 0..20 spherical caves), generated on the device: one
    batched build of all chunks (autotuned) vs the per-chunk loop of plain builds."""
    import torch
    from pyrit_b200 import autotune, gpu_build, native
    from pyrit_b200 import workloads as wl

    from pyrit_b200 import shard

    K = args.chunks
    rank, world, local = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1), _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    L = native.lib()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    ex = native.Exec()
    ex.stream = ctypes.c_void_p(sptr)
    # weak scaling: a world of world*K chunks, each rank builds its contiguous K
    lo, hi = shard.chunk_range(world * K, rank, world)
    log2s = np.ascontiguousarray(wl.chunk_mix(world * K, 0)[lo:hi])
    vox, offs = wl.mix_chunks_device(log2s, lo, 0)
    total = int(offs[-1])
    d_log2 = torch.from_numpy(log2s.view(np.int32)).cuda()
    d_offs = torch.from_numpy(offs.astype(np.uint32).view(np.int32)).cuda()
    counts = torch.zeros(native.COUNTS_WORDS, dtype=torch.int32).pin_memory()
    roots = torch.zeros(K, dtype=torch.int32).pin_memory()
    first = torch.zeros(K, dtype=torch.int32).pin_memory()
    fprim = torch.zeros(K, dtype=torch.int32).pin_memory()

    def batch_desc(k):
        return native.Batch(count=k, log2_host=log2s.ctypes.data, log2=d_log2.data_ptr(), voxels=vox.data_ptr(),
                            voxel_offsets=d_offs.data_ptr(), edits=0, edit_offsets=0,
                            voxel_total=int(offs[k]), edit_total=0)

    def batched_once(k=K):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        bd = batch_desc(k)
        out = native.BuiltC()
        a.record(stream)
        native.check(L.pyrb_build_batch_async(ctypes.byref(ex), ctypes.byref(bd), 5, roots.data_ptr(),
                                              first.data_ptr(), fprim.data_ptr(), counts.data_ptr(),
                                              ctypes.byref(out)))
        b.record(stream)
        L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(out))
        return a, b

    # autotune on the first 128 chunks, then measure the full batch
    best, _ = autotune.sweep(lambda: batched_once(min(128, K)), reps=2, budget_s=args.tune_budget)
    autotune.apply(best)
    for _ in range(2):
        batched_once()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    times = []
    for _ in range(args.batched_reps):
        a, b = batched_once()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    o = native.BuiltC()
    native.check(L.pyrb_build_finish(counts.data_ptr(), ctypes.byref(o)))
    n_u = o.voxel_count
    t_batched = min(times)
    # per-stage CUDA events of one more batched build
    L.pyrb_profile_enable(1)
    try:
        batched_once()
        torch.cuda.synchronize()
        ms = (ctypes.c_float * 256)()
        names = ctypes.create_string_buffer(256 * 32)
        k = L.pyrb_profile_read(ms, names, 32, 256)
        batch_stages = {names.raw[i * 32:(i + 1) * 32].split(b"\0")[0].decode(): round(ms[i], 4)
                        for i in range(min(k, 256))}
    finally:
        L.pyrb_profile_enable(0)

    # chunk install: attribute palettes over the batch (scan + pack), device time
    bd = batch_desc(K)
    out = native.BuiltC()
    native.check(L.pyrb_build_batch(ctypes.byref(ex), ctypes.byref(bd), 5, roots.data_ptr(), first.data_ptr(),
                                    fprim.data_ptr(), ctypes.byref(out)))
    rts, fv = roots.numpy().view(np.uint32), first.numpy().view(np.uint32)
    nz = np.nonzero(rts != 0xFFFFFFFF)[0]
    # every chunk's voxel count as the batch stores it: the root's count word
    from pyrit_b200 import _cudart
    batch_voxels = np.zeros(K, np.uint32)
    one = np.zeros(1, np.uint32)
    for c in nz:
        _cudart.dtoh(one.ctypes.data, out.nodes + 4 * (int(rts[c]) + 1), 4)
        batch_voxels[c] = one[0]
    pfirst = np.concatenate([fv[nz], [out.voxel_count]]).astype(np.uint32)
    pal_t, pack_t = [], []
    for _ in range(3):
        a, b2, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        pal, pcnt = gpu_build.palette_scan(out.attrs, pfirst, stream=sptr)
        b2.record(stream)
        dst, words = gpu_build.palette_layout(pfirst, pcnt)
        pool = torch.empty(max(words, 1), dtype=torch.int32, device="cuda")
        b3 = torch.cuda.Event(enable_timing=True)
        b3.record(stream)
        gpu_build.palette_pack(out.attrs, pfirst, pal, pcnt, dst, pool, stream=sptr)
        c2.record(stream)
        torch.cuda.synchronize()
        pal_t.append(a.elapsed_time(b2))
        pack_t.append(b3.elapsed_time(c2))
        del pool
    path_edit = path_edit_bench(out, rts, fv, fprim.numpy().view(np.uint32), log2s, nz)
    L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(out))
    n_attr = int(pfirst[-1])
    palette = {"chunks": int(len(nz)), "palette_chunks": int((pcnt != 0xFFFFFFFF).sum()),
               "scan_ms": min(pal_t), "pack_ms": min(pack_t), "pool_words": int(words),
               "attr_words": n_attr, "pool_fraction": words / max(n_attr, 1),
               "scan_gbs": 4 * n_attr / (min(pal_t) / 1e3) / 1e9,
               "pack_gbs": (4 * n_attr + 4 * words) / (min(pack_t) / 1e3) / 1e9}

    # per-chunk loop of plain builds (asynchronous, one stream; each chunk's counts land
    # in its own pinned slot)
    loop_counts = torch.zeros((K, native.COUNTS_WORDS), dtype=torch.int32).pin_memory()

    def loop_once():
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for c in range(K):
            out = native.BuiltC()
            n = int(offs[c + 1] - offs[c])
            native.check(L.pyrb_build_async(ctypes.byref(ex), int(log2s[c]), 5, 0, 0, 0,
                                            vox.data_ptr() + 16 * int(offs[c]), n, loop_counts[c].data_ptr(),
                                            ctypes.byref(out)))
            L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(out))
        b.record(stream)
        return a, b

    loop_once()
    torch.cuda.synchronize()
    a, b = loop_once()
    torch.cuda.synchronize()
    t_loop = a.elapsed_time(b)
    # the batch builds what the loop builds: each chunk's voxel count, empty chunks included
    loop_voxels = np.zeros(K, np.uint32)
    for c in range(K):
        f = native.BuiltC()
        native.check(L.pyrb_build_finish(ctypes.c_void_p(loop_counts[c].data_ptr()), ctypes.byref(f)))
        loop_voxels[c] = f.voxel_count
    mismatch = np.nonzero(loop_voxels != batch_voxels)[0]
    assert len(mismatch) == 0, "batched and per-chunk voxel counts differ at chunks %s" % mismatch[:8].tolist()
    comb = shard.combine({"voxels": n_u, "entries": total, "chunks": K, "batched_ms": t_batched, "loop_ms": t_loop})
    n_u, total, t_batched, t_loop = int(comb["voxels"]), int(comb["entries"]), comb["batched_ms"], comb["loop_ms"]
    res = {"chunks": int(comb["chunks"]), "entries": total, "unique_voxels": n_u, "batched_ms": t_batched,
           "batched_voxels_per_s": n_u / (t_batched / 1e3), "per_chunk_loop_ms": t_loop,
           "per_chunk_loop_voxels_per_s": n_u / (t_loop / 1e3), "speedup_vs_per_chunk_loop": t_loop / t_batched,
           "n_gpus": world, "scaling": "weak", "chunks_per_gpu": K, "palette": palette, "path_edit": path_edit,
           "per_chunk_voxels_checked": "nodes[root + 1] of every chunk of the batch equals the voxel count of its "
                                       "plain build in the loop (%d chunks, %d empty)" % (K, K - len(nz)),
           "tuning": {k: best.get(k) for k in ("radix_bits", "tile_keys", "load_factor_pct", "path")},
           "stages_ms": batch_stages,
           "edges": {str(1 << l): int((log2s == l).sum()) for l in (5, 6, 7, 8)}}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if emit and rank == 0:
        print(json.dumps({"metric": METRIC + " (batched, 1024 mixed chunks)", "value": res["batched_voxels_per_s"],
                          "unit": "voxels/s", "n_gpus": world, "higher_is_better": True, "data": "synthetic",
                          "config": {"workload": "batched build of 1024 chunks of the mix, generated on the device"},
                          "batched": res}), flush=True)
    del vox
    torch.cuda.empty_cache()
    return res


def serve_autotune(vox, offs, log2s, budget_s, chunks=64):
    """The autotuner on a served-size batch (the first `chunks` chunks of the pool): the
    setting it finds stays applied for the serving that follows."""
    import torch
    from pyrit_b200 import autotune, native
    L = native.lib()
    stream = torch.cuda.current_stream()
    ex = native.Exec()
    ex.stream = ctypes.c_void_p(stream.cuda_stream)
    k = min(chunks, len(log2s))
    lg = np.ascontiguousarray(log2s[:k], dtype=np.uint32)
    d_lg = torch.from_numpy(lg.view(np.int32)).cuda()
    o32 = np.ascontiguousarray(offs[:k + 1], dtype=np.uint32)
    d_off = torch.from_numpy(o32.view(np.int32)).cuda()
    counts = torch.zeros(native.COUNTS_WORDS, dtype=torch.int32).pin_memory()
    res = torch.zeros(k, dtype=torch.int32).pin_memory()

    def once():
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        bd = native.Batch(count=k, log2_host=lg.ctypes.data, log2=d_lg.data_ptr(), voxels=vox.data_ptr(),
                          voxel_offsets=d_off.data_ptr(), edits=0, edit_offsets=0, voxel_total=int(o32[-1]),
                          edit_total=0)
        out = native.BuiltC()
        a.record(stream)
        native.check(L.pyrb_build_batch_async(ctypes.byref(ex), ctypes.byref(bd), 5, res.data_ptr(), res.data_ptr(),
                                              res.data_ptr(), counts.data_ptr(), ctypes.byref(out)))
        b.record(stream)
        L.pyrb_built_free(ctypes.byref(ex), ctypes.byref(out))
        return a, b

    best, _ = autotune.sweep(once, reps=2, budget_s=budget_s)
    autotune.apply(best)
    return {x: best.get(x) for x in ("radix_bits", "tile_keys", "load_factor_pct", "path")}


def run_served(args, emit=True):
    """Poisson arrivals of chunk-build requests (a chunk of the 1024-chunk mix plus 0..64
    random edits) at --rate per second for --duration seconds, served by continuous
    batching (the library's native served loop, pyrb_server_*) with a 40 GB budget for
    dedup tables, scratch and the DAG arena."""
    import torch
    from pyrit_b200 import workloads as wl
    from pyrit_b200.serve import ChunkPool, ChunkServer, Request

    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    K = args.chunks
    log2s = wl.chunk_mix(K, 0)
    vox, offs = wl.mix_chunks_device(log2s, 0, 0)
    pool = ChunkPool(vox, offs, log2s)
    tuning = serve_autotune(vox, offs, log2s, args.tune_budget)
    out = {}
    for rate in args.rates:
        n = int(rate * args.duration)
        arr = wl.poisson_arrivals(n, rate, 7)
        rng = np.random.default_rng(11)
        chunks = rng.integers(0, K, n)
        nedits = rng.integers(0, 65, n)
        reqs = [Request(i, int(chunks[i]), wl.chunk_edits(int(log2s[chunks[i]]), int(nedits[i]), 5000 + i),
                        float(arr[i])) for i in range(n)]
        srv = ChunkServer(pool, budget_bytes=40 << 30, max_batch_voxels=args.max_batch_voxels,
                          max_inflight=args.max_inflight, rt_log2=5)
        srv.keep_results = False
        # warm-up on a few requests (not timed)
        srv.serve([Request(-1 - i, int(chunks[i]), reqs[i].edits, 0.0) for i in range(4)], realtime=False)
        srv.release_all()
        st = srv.serve(reqs, realtime=True)
        srv.release_all()
        srv.close()
        s = st.summary()
        s["offered_req_per_s"] = rate
        s["offered_voxels_per_s"] = float(np.mean(pool.sizes[chunks]) * rate)
        out[str(int(rate))] = s
    if emit:
        print(json.dumps({"metric": METRIC + " (served, Poisson arrivals)", "unit": "voxels/s", "n_gpus": 1,
                          "higher_is_better": True, "data": "synthetic",
                          "config": {"workload": "Poisson chunk requests from the 1024-chunk mix + 0..64 edits",
                                     "duration_s": args.duration, "budget_gb": 40,
                                     "max_batch_voxels": args.max_batch_voxels, "max_inflight": args.max_inflight},
                          "tuning": tuning, "served": out}), flush=True)
    del vox
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["noise256", "bernoulli1024", "bernoulli512", "batched", "served", "worst"],
                    default="noise256")
    ap.add_argument("--rates", type=float, nargs="+", default=[20000.0])
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--max-batch-voxels", type=int, default=32 << 20)
    ap.add_argument("--max-inflight", type=int, default=2)
    ap.add_argument("--chunks", type=int, default=1024)
    ap.add_argument("--batched-reps", type=int, default=3)
    ap.add_argument("--tune-budget", type=float, default=15.0)
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: skip the batched, served and worst-case objects")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        run_batched(args)
        return 0
    if args.workload == "served":
        run_served(args)
        return 0
    if args.workload == "worst":
        import torch
        torch.cuda.set_device(_env_int("LOCAL_RANK", 0))
        print(json.dumps({"metric": METRIC + " (worst case)", "unit": "voxels/s", "n_gpus": 1,
                          "worst_case": run_worst_case(args)}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
