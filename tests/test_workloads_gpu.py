"""The device-side chunk-mix generator yields exactly the host generator's voxel lists."""
import numpy as np
import pytest

from pyrit_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def test_device_mix_matches_host():
    log2s = np.array([5, 6, 5, 7, 6, 5], np.uint32)
    vox, offs = wl.mix_chunks_device(log2s, 3, 0)
    v = vox.cpu().numpy().view(np.uint32)
    for c, l in enumerate(log2s):
        ref = wl.mix_chunk(3 + c, int(l), 0)
        assert np.array_equal(v[offs[c]:offs[c + 1]], ref), c
