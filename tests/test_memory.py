"""Device memory of a build, from the host-side bounds the build allocates from
(pyrb_build_memory; host only, no GPU). The reference caps the peak allocation of its
GPU build at 130 bytes per voxel (tests/cpu_test.zig:1559-1629, measured with a
counting Exec); the same cap holds here for the plain 256^3 noise build with its edit
overlay and for the 1024^3 worst case, where the bounds, taken from the input size,
are tight. The GPU suite checks that a real build reports the same bytes."""
import numpy as np
import pytest

from pyrit_b200 import gpu_build, native

# (edge log2, entries) of the plain 256^3 noise + 0.5 % edits and the 1024^3
# Bernoulli(0.15) + 10^6 edits workloads
DENSE_CONFIGS = [(8, 5_116_905), (10, 162_054_872)]


@pytest.mark.parametrize("log2,entries", DENSE_CONFIGS)
def test_bytes_per_entry_below_the_reference_cap(log2, entries):
    scratch, outputs = gpu_build.build_memory(log2, entries, rt_log2_req=7)
    assert scratch > 0 and outputs > 0
    assert (scratch + outputs) / entries < 130


def test_bounds_grow_with_the_input():
    s1, o1 = gpu_build.build_memory(8, 100_000)
    s2, o2 = gpu_build.build_memory(8, 200_000)
    assert s2 > s1 and o2 > o1
    # chunks of the same edge: more cells bound the upper levels
    sc, oc = gpu_build.build_memory(6, 200_000, count=8)
    assert sc > 0 and oc > 0
    # a batch of mixed edges
    sb, ob = gpu_build.build_memory(0, 3_000_000, chunk_log2=[5, 6, 7, 8])
    assert sb > 0 and ob > 0


def test_invalid_requests_are_rejected():
    for args in [(2, 1000), (21, 1000), (8, 1 << 31)]:
        with pytest.raises(native.PyrbError) as e:
            gpu_build.build_memory(*args)
        assert e.value.code == native.PYRB_ERROR_INVALID_ARGUMENT
    with pytest.raises(native.PyrbError):
        gpu_build.build_memory(8, 1000, count=0)
    with pytest.raises(native.PyrbError):
        gpu_build.build_memory(0, 1000, chunk_log2=np.array([5, 2], np.uint32))
