"""GPU: kspn_normalise_noalloc, the relabel entry point that allocates
nothing, called through the C ABI and checked against kspn_normalise (the
context-based entry point) on the same ids, two calls in a row.

It serves callers that cannot call cudaMalloc when they need the relabel
(device memory already handed out by their own pool allocator, or no room
for the synchronisation an allocation may cause); its scratch is a fixed
device array for at most KSPN_NOALLOC_MAX_N vertices.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it passes alone and after the others."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O
from kspn_testlib import dev_to_u32, u32_to_dev

pytestmark = pytest.mark.gpu


def test_noalloc_relabel_matches_context_entry_point():
    import torch

    L = K.lib()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    with K.Context(0) as ctx:
        # the largest allowed n first, then a smaller one: the second call
        # must not see what the first left in the shared array
        for n in (K.NOALLOC_MAX_N, 1000, 1000):
            ids = rng.integers(0, n, n).astype(np.uint32)
            want = u32_to_dev(ids)
            got = u32_to_dev(ids)
            torch.cuda.synchronize()
            ctx.normalise(n, want)
            rc = L.kspn_normalise_noalloc(n, C.c_void_p(got.data_ptr()), C.c_void_p(stream.cuda_stream))
            assert rc == 0, K.STATUS.get(rc, rc)
            assert np.array_equal(dev_to_u32(got)[:n], dev_to_u32(want)[:n])
            assert np.array_equal(dev_to_u32(got)[:n], O.normalise(ids))


def test_noalloc_relabel_rejects_too_many_vertices():
    import torch

    L = K.lib()
    buf = torch.zeros(8, dtype=torch.int32, device="cuda")
    assert L.kspn_normalise_noalloc(K.NOALLOC_MAX_N + 1, C.c_void_p(buf.data_ptr()), None) == 1
    assert L.kspn_normalise_noalloc(0, None, None) == 0


def test_noalloc_relabel_reports_out_of_range_id():
    """An id >= n is KSPN_ERR_INVALID_ARGUMENT; the array is then partly
    relabelled: that id is unchanged and every id < n is already replaced
    by the smallest vertex carrying it.  The next call is unaffected."""
    import torch

    L = K.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = 5000
    ids = np.random.default_rng(3).integers(0, n, n).astype(np.uint32)
    ids[123] = n + 7
    got = u32_to_dev(ids)
    torch.cuda.synchronize()
    assert L.kspn_normalise_noalloc(n, C.c_void_p(got.data_ptr()), stream) == 1
    valid = ids < n
    first = np.full(n, 0xFFFFFFFF, np.uint32)
    np.minimum.at(first, ids[valid], np.nonzero(valid)[0].astype(np.uint32))
    want = ids.copy()
    want[valid] = first[ids[valid]]
    assert np.array_equal(dev_to_u32(got)[:n], want)
    ok = np.random.default_rng(4).integers(0, n, n).astype(np.uint32)
    got = u32_to_dev(ok)
    torch.cuda.synchronize()
    assert L.kspn_normalise_noalloc(n, C.c_void_p(got.data_ptr()), stream) == 0
    assert np.array_equal(dev_to_u32(got)[:n], O.normalise(ok))
