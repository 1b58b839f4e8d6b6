"""Minimal CUDA runtime access (ctypes) for host<->device copies of raw device addresses."""
from __future__ import annotations

import ctypes
import glob
import os

_rt = None


def rt():
    global _rt
    if _rt is None:
        cands = []
        try:
            import nvidia  # noqa: F401  (torch's bundled runtime, already loaded by torch)
            base = os.path.dirname(nvidia.__path__[0])
            cands += glob.glob(os.path.join(base, "nvidia", "cuda_runtime", "lib", "libcudart.so.12"))
        except Exception:
            pass
        cands += ["libcudart.so.12", "/usr/local/cuda/lib64/libcudart.so.12"]
        last = None
        for c in cands:
            try:
                _rt = ctypes.CDLL(c)
                break
            except OSError as e:
                last = e
        if _rt is None:
            raise RuntimeError(f"libcudart not found: {last}")
        _rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        _rt.cudaMemcpy.restype = ctypes.c_int
    return _rt


def dtoh(dst_ptr: int, src_addr: int, nbytes: int) -> None:
    if nbytes:
        rc = rt().cudaMemcpy(ctypes.c_void_p(dst_ptr), ctypes.c_void_p(src_addr), nbytes, 2)
        if rc != 0:
            raise RuntimeError(f"cudaMemcpy DtoH failed ({rc})")


def htod(dst_addr: int, src_ptr: int, nbytes: int) -> None:
    if nbytes:
        rc = rt().cudaMemcpy(ctypes.c_void_p(dst_addr), ctypes.c_void_p(src_ptr), nbytes, 1)
        if rc != 0:
            raise RuntimeError(f"cudaMemcpy HtoD failed ({rc})")


def dtod(dst_addr: int, src_addr: int, nbytes: int) -> None:
    if nbytes:
        rc = rt().cudaMemcpy(ctypes.c_void_p(dst_addr), ctypes.c_void_p(src_addr), nbytes, 3)
        if rc != 0:
            raise RuntimeError(f"cudaMemcpy DtoD failed ({rc})")
