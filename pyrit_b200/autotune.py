"""Autotuner of the build's ordering path, sort and dedup parameters.

Sweeps the way voxels are ordered (the cell grid, the brick buckets, or the radix sort
with its digit width of 4, 8, 9, 10, 11 bits and keys per sort tile of 1024, 2048,
4096, or 8192 with 8- or 9-bit digits) and the dedup hash-table load factor (50 %, 70 %) on a
caller-supplied workload, times every setting with CUDA events, applies the fastest
through pyrb_set_tuning and can persist it as JSON. None of the parameters changes
the output (the build is bit-exact for all of them); they only change speed and
memory. The grid and bucket settings come first (four of them); the sort settings
follow while the time budget lasts.
"""
from __future__ import annotations

import itertools
import json
import os
import time

from . import gpu_build, native

RADIX_BITS = (4, 8, 9, 10, 11)
TILE_KEYS = (1024, 2048, 4096, 8192)
LOAD_FACTORS = (50, 70)


def supported(radix_bits: int, tile_keys: int) -> bool:
    """8192-entry sort tiles exist for 8- and 9-bit digits only."""
    return tile_keys != 8192 or radix_bits in (8, 9)


def default_path() -> str:
    return os.path.join(os.path.expanduser("~"), ".cache", "pyrit_b200", "tuning.json")


def sweep(run_once, reps: int = 3, radix_bits=RADIX_BITS, tile_keys=TILE_KEYS, load_factors=LOAD_FACTORS,
          budget_s: float = 60.0):
    """run_once() must enqueue one build on the current stream and return a pair of
    (start, end) CUDA events around it. Returns (best setting, all results)."""
    import torch
    old = gpu_build.get_tuning()
    results = []
    if budget_s <= 0:   # no sweep: report the current setting
        cur = {"radix_bits": old.radix_bits, "tile_keys": old.tile_keys, "load_factor_pct": old.load_factor_pct,
               "path": old.path, "ms": None}
        return cur, [cur]
    t_start = time.time()
    settings = [(0, 0, lf, path) for path in (native.PATH_GRID, native.PATH_BUCKET) for lf in load_factors] + [
        (rb, tk, lf, native.PATH_SORT) for rb, tk, lf in itertools.product(radix_bits, tile_keys, load_factors)
        if supported(rb, tk)]
    try:
        for rb, tk, lf, path in settings:
            if time.time() - t_start > budget_s:
                break
            gpu_build.set_tuning(rb, tk, lf, path)
            run_once()  # warm-up of this setting
            torch.cuda.synchronize()
            times = []
            for _ in range(reps):
                a, b = run_once()
                torch.cuda.synchronize()
                times.append(a.elapsed_time(b))
            results.append({"radix_bits": rb, "tile_keys": tk, "load_factor_pct": lf, "path": path,
                            "ms": min(times)})
    finally:
        gpu_build.set_tuning(old.radix_bits, old.tile_keys, old.load_factor_pct, old.path)
    best = min(results, key=lambda r: r["ms"])
    return best, results


def apply(setting: dict) -> None:
    gpu_build.set_tuning(setting["radix_bits"], setting["tile_keys"], setting["load_factor_pct"],
                         setting.get("path", native.PATH_AUTO))


def save(setting: dict, path: str | None = None) -> str:
    path = path or default_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump(setting, f)
    return path


def load(path: str | None = None) -> dict | None:
    path = path or default_path()
    if not os.path.exists(path):
        return None
    with open(path) as f:
        s = json.load(f)
    apply(s)
    return s
