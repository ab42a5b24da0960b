"""The Python glue of the updatable indexes' searches, up to the library call
(no GPU): the C entry point and the device mirror's search are replaced by
stand-ins that record what they were given.  Checks that batches reach the
library as f32[nq, dim] with nq as given, that the per-query wrappers
unpack counts and ids, and that wrong-length queries never get there."""
import threading

import numpy as np
import pytest

import pydiskann_b200.incremental as inc_mod
import pydiskann_b200.spfresh as spf_mod
from pydiskann_b200.incremental import DELTA_ID_OFFSET, IncrementalDiskANN
from pydiskann_b200.spfresh import SPFresh


class FakeSpfLib:
    """dg_spfresh_search_batch: query i gets ids 10i, 10i+1, ... (i + 1 of them, at most k)."""

    def __init__(self):
        self.calls = []

    def dg_spfresh_search_batch(self, h, p, q, nq, out_ids, out_d, out_cnt):
        import ctypes as C

        k = p._obj.k
        self.calls.append((nq, k))
        ids = np.ctypeslib.as_array(C.cast(out_ids, C.POINTER(C.c_uint64)), (nq, k))
        ds = np.ctypeslib.as_array(C.cast(out_d, C.POINTER(C.c_float)), (nq, k))
        cnt = np.ctypeslib.as_array(C.cast(out_cnt, C.POINTER(C.c_uint32)), (nq,))
        for i in range(nq):
            c = min(i + 1, k)
            cnt[i] = c
            ids[i, :c] = 10 * i + np.arange(c)
            ds[i, :c] = np.arange(c, dtype=np.float32) / 2
        return 0


def test_spfresh_search_glue(monkeypatch):
    fake = FakeSpfLib()
    monkeypatch.setattr(spf_mod, "lib", lambda: fake)
    s = SPFresh(4, device=None)
    s._h = object()  # stands in for the device mirror
    try:
        assert s.search_batch(np.zeros((3, 4), np.float32), k=2, n_probe=5) == [[0], [10, 11], [20, 21]]
        assert fake.calls[-1] == (3, 2)
        assert s.search_with_dists([0.0] * 4, k=3) == [(0, 0.0)]
        for bad in ([0.0] * 8, np.zeros((2, 3)), [[0.0] * 4, [0.0] * 3]):
            with pytest.raises(ValueError, match="Query dim"):
                s.search_batch(bad, k=2)
        assert len(fake.calls) == 2
    finally:
        s._h = None


def test_incremental_search_glue(monkeypatch):
    seen = []

    def fake_search(ix, Q, k, L, traversal, rerank_size, filters):
        seen.append((Q.shape, Q.dtype, k, L))
        nq = len(Q)
        ids = np.full((nq, k), 0xFFFFFFFF, np.uint32)
        ids[:, 0] = np.arange(nq) + 5  # delta rows: base_count is 5
        ids[:, 1] = np.arange(nq)
        return ids, np.zeros((nq, k), np.float32), np.full(nq, 2, np.uint32)

    monkeypatch.setattr(inc_mod, "_mirror_search", fake_search)
    o = object.__new__(IncrementalDiskANN)
    o._lock = threading.RLock()
    o.dim, o._nf, o.quantizer, o.rerank_size, o._ix = 4, 0, None, 0, None
    o._bX = np.zeros((5, 4), np.float32)
    got = o.search_batch(np.ones((3, 4)), k=4, beam_width=16)
    assert seen[-1] == ((3, 4), np.float32, 4, 16)
    assert got == [[DELTA_ID_OFFSET + i, i] for i in range(3)]
    assert o.search([0.0] * 4, k=4) == [DELTA_ID_OFFSET, 0]
    for bad in ([0.0] * 8, np.zeros((2, 3))):
        with pytest.raises(ValueError, match="Query dim"):
            o.search_batch(bad, k=2)
    assert len(seen) == 2
