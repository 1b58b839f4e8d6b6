"""Compiles the native libraries in-tree.

* ``pyrit_b200/libpyrit_b200.so``  -- the CUDA DAG build for sm_100a behind the
  C ABI of ``include/pyrit_b200.h`` (nvcc, ``-gencode arch=compute_100a,code=sm_100a``).
* ``pyrit_b200/libpyrb_workloads.so`` -- seeded synthetic workload generators (host C++).

Run ``python -m pyrit_b200._build`` or call :func:`build_all`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

CUDA_SOURCES = ["pyrb_build.cu", "pyrb_server.cpp"]
# every header next to the sources: a change to any of them rebuilds the library
CUDA_HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")) and not f.startswith("workloads"))
WORKLOAD_SOURCES = ["workloads.cpp", "workloads_gpu.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-shared",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA build needs nvcc 12.8+ for sm_100a")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: " + " ".join(cmd))


def build_cuda(force: bool = False, verbose_ptxas: bool = False) -> str:
    out = os.path.join(HERE, "libpyrit_b200.so")
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [os.path.join(INCLUDE, "pyrit_b200.h")]
    if force or _stale(out, deps):
        cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-o", out, *srcs]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
    return out


def build_workloads(force: bool = False) -> str:
    """Workload generators: host C++ (g++) plus the device-side chunk-mix generator (nvcc)."""
    out = os.path.join(HERE, "libpyrb_workloads.so")
    srcs = [os.path.join(CSRC, s) for s in WORKLOAD_SOURCES]
    deps = srcs + [os.path.join(CSRC, "workloads.h")]
    if force or _stale(out, deps):
        _run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-pthread", "-Xcompiler", "-ffp-contract=off",
              "-I", CSRC, "-o", out, *srcs])
    return out


def build_all(force: bool = False) -> None:
    build_workloads(force)
    build_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
