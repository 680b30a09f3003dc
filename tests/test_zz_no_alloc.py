"""The allocation-free ordering entry point (pggc_generate_orderings_noalloc).

It exists for callers that cannot allocate device memory (a framework that
owns all device memory, an allocator-free loop):
its scratch is a fixed array inside the library.  Checked through the C ABI
against the allocating pggc_generate_orderings on two calls in a row with
different graphs, so stale scratch from the first call would show up in the
second.  Collected last so a failure here does not hide other tests.
"""
import ctypes

import numpy as np
import pytest

import pennsylvaniagpugraphclustering_b200 as pg
from pennsylvaniagpugraphclustering_b200 import _lib

from . import graphs as G

pytestmark = pytest.mark.gpu

MAX_N = 16 * 1024 * 1024


def _noalloc(hg):
    import torch
    rowptr = torch.from_numpy(hg.rowptr).cuda()
    o1 = torch.full((max(hg.n, 1),), -7, dtype=torch.int32, device="cuda")
    o2 = torch.full((max(hg.n, 1),), -7, dtype=torch.int32, device="cuda")
    off = torch.full((4,), -7, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().pggc_generate_orderings_noalloc(rowptr.data_ptr(), hg.n, o1.data_ptr(), o2.data_ptr(),
                                                          off.data_ptr(), ctypes.c_void_p(stream)))
    torch.cuda.synchronize()
    return o1.cpu().numpy()[:hg.n], o2.cpu().numpy()[:hg.n], off.cpu().numpy()


def _regular(mem, hg):
    wg = pg.weighted_graph(mem, hg.rowptr, hg.col)
    return pg.generate_orderings(mem, wg)


def test_noalloc_matches_allocating_entry_point_twice():
    mem = pg.memory_store(0)
    first = G.hub_graph()            # all three degree buckets, 16,001 vertices
    second = G.small_rmat(seed=3)    # smaller: stale counts from the first call would show
    for hg in (first, second):
        a1, a2, aoff = _noalloc(hg)
        r1, r2, roff = _regular(mem, hg)
        assert np.array_equal(a1, r1)
        assert np.array_equal(a2, r2)
        assert np.array_equal(aoff, roff)


def test_noalloc_rejects_oversized_graph():
    import torch
    dummy = torch.zeros(8, dtype=torch.int64, device="cuda")
    st = _lib.lib().pggc_generate_orderings_noalloc(dummy.data_ptr(), MAX_N + 1, dummy.data_ptr(), dummy.data_ptr(),
                                                    dummy.data_ptr(), None)
    assert st == _lib.PGGC_ERR_INVALID
    assert b"16,777,216" in _lib.lib().pggc_last_error()
