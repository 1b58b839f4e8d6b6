"""The C-ABI library loads and exports every symbol that include/pyrit_b200.h declares
(CPU only: no compute call is made)."""
import ctypes
import os
import re

from pyrit_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"PYRB_API\s+[\w\s\*]+?\b(pyrb_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert {"pyrb_build", "pyrb_build_chunks", "pyrb_downsample", "pyrb_built_free"} <= names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(native.LIB_PATH):
        from pyrit_b200 import _build
        _build.build_cuda()
    lib = ctypes.CDLL(native.LIB_PATH)
    missing = [n for n in sorted(_declared_symbols()) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_header():
    assert _declared_symbols() <= set(native.SIGNATURES)


def test_host_only_calls():
    L = native.lib()
    assert L.pyrb_version() >= 1
    assert L.pyrb_result_string(-1) == b"invalid argument"
    t = native.Tuning(radix_bits=5, tile_keys=4096, load_factor_pct=50)  # 5 is not a supported width
    assert L.pyrb_set_tuning(ctypes.byref(t)) == -1
    assert b"radix_bits" in L.pyrb_error_message()
    t = native.Tuning(radix_bits=10, tile_keys=8192, load_factor_pct=50)  # 8192-entry tiles take 8 or 9 bits
    assert L.pyrb_set_tuning(ctypes.byref(t)) == -1
    assert b"8192" in L.pyrb_error_message()
    t = native.Tuning(radix_bits=0, tile_keys=4096, load_factor_pct=50)  # automatic is both or neither
    assert L.pyrb_set_tuning(ctypes.byref(t)) == -1
    t = native.Tuning(radix_bits=0, tile_keys=0, load_factor_pct=50)
    assert L.pyrb_set_tuning(ctypes.byref(t)) == 0
    g = native.Tuning()
    L.pyrb_get_tuning(ctypes.byref(g))
    assert (g.radix_bits, g.tile_keys, g.load_factor_pct) == (0, 0, 50)


def test_struct_layouts():
    # pyrb_built mirrors gpu_build.Built with explicit padding (88 bytes)
    assert ctypes.sizeof(native.BuiltC) == 88
    assert ctypes.sizeof(native.ChunkBatch) == 32
    assert ctypes.sizeof(native.Exec) == 32


def test_autotune_offers_only_supported_settings():
    """8192-entry tiles exist for 8- and 9-bit digits only; the sweep skips the rest."""
    from pyrit_b200 import autotune
    assert 8192 in autotune.TILE_KEYS
    offered = [(rb, tk) for rb in autotune.RADIX_BITS for tk in autotune.TILE_KEYS if autotune.supported(rb, tk)]
    assert (9, 8192) in offered and (8, 8192) in offered
    assert all(tk != 8192 or rb in (8, 9) for rb, tk in offered)
    L = native.lib()
    for rb, tk in offered:  # every offered setting is accepted by the library
        t = native.Tuning(radix_bits=rb, tile_keys=tk, load_factor_pct=50)
        assert L.pyrb_set_tuning(ctypes.byref(t)) == 0
    t = native.Tuning(radix_bits=0, tile_keys=0, load_factor_pct=50)
    assert L.pyrb_set_tuning(ctypes.byref(t)) == 0
