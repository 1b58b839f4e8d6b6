"""Device-side error paths, provoked without faulting or hanging the GPU.

* A bounded wait that nothing ends (pyrb_selftest_wait_limit: a look-back whose
  predecessor never publishes) gives up after its poll limit, sets the error word and
  returns: the call reports PYRB_ERROR_CUDA with the wait-limit message, as a build
  would, and the context stays usable (a build right after is bit-exact).
* The world path never cuts a chunk off: a generator count above the capacity is
  reported as PYRB_ERROR_CAPACITY with the count needed (the reference grows the
  capacity and generates again, src/world.zig:968-996); the retry with the grown
  capacity builds what the reference's worldedit + buildChunks would."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc
from pyrit_b200 import native
from pyrit_b200 import workloads as wl

from gpu_helpers import assert_same_build, dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, 1])
def test_wait_limit_is_reported_and_the_context_survives(which):
    import torch
    from pyrit_b200 import gpu_build
    L = native.lib()
    ex = native.Exec()
    ex.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.pyrb_selftest_wait_limit(ctypes.byref(ex), which)
    assert rc == native.PYRB_ERROR_CUDA
    assert b"look-back wait limit" in L.pyrb_error_message()
    pts = wl.heightfield(6, 1)
    g = gpu_build.build(6, 4, dev(pts)).download()
    assert_same_build(g, orc.gb_build(6, 4, pts), label="after the wait limit")


def _world_inputs(K, log2, cap, counts_wanted, seed):
    rng = np.random.default_rng(seed)
    n = 1 << log2
    vox = np.zeros((K * cap, 4), np.uint32)
    counts = np.zeros(K, np.uint32)
    gens = []
    for c in range(K):
        g = wl.mix_chunk(400 + c, log2, seed)[:counts_wanted[c]]
        gens.append(g)
        k = min(len(g), cap)  # a generator writes at most `capacity` voxels, but counts them all
        vox[c * cap:c * cap + k] = g[:k]
        counts[c] = len(g)
    edits, eoff = [], [0]
    for c in range(K):
        pos = rng.choice(n ** 3, int(rng.integers(0, 200)), replace=False)
        for p in pos:
            edits.append([p % n, (p // n) % n, p // (n * n), 0 if rng.integers(2) else int(rng.integers(1, 9))])
        eoff.append(len(edits))
    return gens, vox, counts, np.array(edits, np.uint32).reshape(-1, 4), np.array(eoff, np.uint32)


def test_chunk_over_capacity_is_reported_and_the_retry_builds_everything():
    from pyrit_b200 import gpu_build
    K, log2, cap = 5, 5, 4000
    want = [3000, 6500, 0, 3900, 5200]
    gens, vox, counts, edits, eoff = _world_inputs(K, log2, cap, want, 3)
    need = int(max(len(g) for g in gens))
    assert need > cap
    with pytest.raises(native.PyrbError) as e:
        gpu_build.build_chunks_edits(log2, 4, K, cap, dev(vox), dev(counts), dev(edits), dev(eoff), int(eoff[-1]))
    assert e.value.code == native.PYRB_ERROR_CAPACITY
    assert gpu_build.last_capacity_need() == need
    # grow the capacity past the need (room for the edits the overlay appends, as the
    # reference's second buffer needs), generate again (here: lay the same lists out
    # again), retry
    cap2 = need + 256
    vox2 = np.zeros((K * cap2, 4), np.uint32)
    for c in range(K):
        vox2[c * cap2:c * cap2 + len(gens[c])] = gens[c]
    g = gpu_build.build_chunks_edits(log2, 4, K, cap2, dev(vox2), dev(counts), dev(edits), dev(eoff),
                                     int(eoff[-1])).download()
    ov, oc = orc.we_apply_all(K, cap2, vox2, counts, edits, eoff)
    offs = np.concatenate([[0], np.cumsum(oc)]).astype(np.uint32)
    packed = np.zeros_like(ov)
    for c in range(K):
        packed[c * cap2:c * cap2 + oc[c]] = ov[c * cap2:c * cap2 + oc[c]]
    o = orc.gb_build_chunks(log2, 4, cap2, packed, offs)
    assert_same_build(g, o, chunks=True, label="grown capacity")
