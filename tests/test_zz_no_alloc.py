"""cirrus_leaf_dot_noalloc, the allocation-free LEAF dot product, against cirrus_dot.

The entry point keeps its reduction scratch in a static device array; two calls in a row must
each give cirrus_dot's bits (the ticket counter is re-armed per call), also after other data
went through the same scratch.  The test itself uploads the leaf list with torch; the entry
point allocates nothing."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cirrus_b200 import LEAF, DeviceGrid, _native

INVALID_ARGUMENT = 1


def _call(a_ptr, b_ptr, leaves_ptr, n_leaf, stream=None):
    out = C.c_double(float("nan"))
    st = _native.lib().cirrus_leaf_dot_noalloc(a_ptr, b_ptr, leaves_ptr, n_leaf, C.byref(out), stream)
    return st, out.value


def test_noalloc_rejects_bad_arguments_before_touching_a_device():
    # argument checks come first, so these run without a GPU
    assert _call(None, None, None, 4)[0] == INVALID_ARGUMENT
    assert _call(C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), -1)[0] == INVALID_ARGUMENT
    assert _call(C.c_void_p(16), C.c_void_p(16), None, 8)[0] == INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sphere64_small", "ring512"])
def test_noalloc_dot_matches_cirrus_dot_twice(name, built_cache):
    import torch

    b = built_cache(name)
    g = DeviceGrid(b.topology)
    leaves = np.flatnonzero(g.tiles[:, 4] & LEAF).astype(np.int32)
    d_leaves = torch.from_numpy(leaves).cuda()
    torch.cuda.synchronize()
    rng = np.random.default_rng(7)
    pa, pb = C.c_void_p(g.channel_ptr(2)), C.c_void_p(g.channel_ptr(3))
    for trial in range(2):
        g.set_channel(2, rng.standard_normal((g.num_tiles, 512)).astype(np.float32))
        g.set_channel(3, rng.standard_normal((g.num_tiles, 512)).astype(np.float32))
        want = g.dot(2, 3)
        got = [_call(pa, pb, C.c_void_p(d_leaves.data_ptr()), len(leaves)) for _ in range(2)]
        for st, v in got:
            assert st == 0
            assert np.float64(v).tobytes() == np.float64(want).tobytes(), (trial, v, want)
    # a dot of a channel with itself: positive, and again equal to cirrus_dot
    st, v = _call(pa, pa, C.c_void_p(d_leaves.data_ptr()), len(leaves))
    assert st == 0 and v > 0 and v == g.dot(2, 2)
    g.close()
