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


def _read(p, dtype, n):
    import ctypes as C

    if not p:
        return None
    return np.frombuffer((C.c_char * (n * np.dtype(dtype).itemsize)).from_address(int(p)), dtype=dtype).copy()


def test_search_params_packing():
    """_Index._params (every host-side search and the autotuner): per-query
    filter programs arrive as ops + offsets[nq + 1] + one value pool, one
    program as ops without offsets, Filter.none() as no program, and one beam
    width per query -- never fewer (the library reads nq of them)."""
    import pydiskann_b200 as dg
    from pydiskann_b200 import Filter

    op_dt = np.dtype({"names": ["op", "field", "a", "b"], "formats": [np.uint32, np.uint32, np.uint64, np.uint64],
                      "offsets": [0, 4, 8, 16], "itemsize": 24})
    ix = object.__new__(dg._Index)
    ix._X = np.zeros((1, 4), np.float32)  # dim 4; nothing reaches a device
    Q = np.zeros((3, 4), np.float32)
    fl = [Filter.in_(0, [5, 6]), Filter.none(), Filter.or_([Filter.eq(1, 2), Filter.in_(2, [9])])]
    p, _, nq, _, _, keep = ix._params(Q, 10, 32, 0, 0, fl, [8, 16, 24], None, None, False)
    offs = _read(p.filter_offsets, np.uint32, nq + 1)
    ops = _read(p.filter_ops, op_dt, int(offs[-1]))
    pool = _read(p.filter_pool, np.uint64, p.filter_pool_len)
    for q, f in enumerate(fl):
        mine = [tuple(int(x) for x in o) for o in ops[offs[q]:offs[q + 1]]]
        want, wpool = f.program()
        assert len(mine) == len(want)
        for (op, field, a, b), (wop, wfield, wa, wb) in zip(mine, want):
            assert (op, field) == (wop, wfield)
            if op == 2:  # IN: offsets rebased into the shared pool
                assert pool[a:a + b].tolist() == wpool[wa:wa + wb]
            else:
                assert (a, b) == (wa, wb)
    assert _read(p.per_query_beam, np.uint32, 3).tolist() == [8, 16, 24]
    p1, *_ = ix._params(Q, 10, 32, 0, 0, Filter.eq(0, 1), None, None, None, False)
    assert p1.filter_nops == 1 and not p1.filter_offsets
    p0, *_ = ix._params(Q, 10, 32, 0, 0, Filter.none(), None, None, None, False)
    assert p0.filter_nops == 0 and not p0.filter_ops
    with pytest.raises(ValueError, match="one beam width per query"):
        ix._params(Q, 10, 32, 0, 0, None, [8, 16], None, None, False)
    with pytest.raises(ValueError, match="one filter per query"):
        ix._params(Q, 10, 32, 0, 0, fl[:2], None, None, None, False)


def test_out_buffers_are_checked():
    """Result buffers given by the caller must hold what the library writes:
    nq * k ids and distances and nq counts, 4 bytes each, contiguous."""
    import pydiskann_b200 as dg

    ix = object.__new__(dg._Index)
    ix._X = np.zeros((1, 4), np.float32)
    Q = np.zeros((3, 4), np.float32)
    good = (np.empty((3, 10), np.uint32), np.empty((3, 10), np.float32), np.empty(3, np.uint32))
    assert ix._params(Q, 10, 32, 0, 0, None, None, good, None, False)[3] is good
    bad = [(np.empty((3, 9), np.uint32), good[1], good[2]), (good[0], np.empty((3, 10), np.float64), good[2]),
           (good[0], good[1], np.empty(2, np.uint32)), (good[0], np.empty((10, 3), np.float32).T, good[2])]
    for out in bad:
        with pytest.raises(ValueError, match="must be a writable contiguous host array"):
            ix._params(Q, 10, 32, 0, 0, None, None, out, None, False)


class _AsCuda:
    """A CPU tensor that reports itself as CUDA, to reach the device-query
    checks, which run before anything is allocated or launched."""

    is_cuda = True

    def __init__(self, t):
        self.t = t

    def data_ptr(self):
        return self.t.data_ptr()

    def contiguous(self):
        return self

    def dim(self):
        return self.t.dim()

    def reshape(self, *s):
        return _AsCuda(self.t.reshape(*s))

    @property
    def shape(self):
        return self.t.shape

    @property
    def dtype(self):
        return self.t.dtype


def test_device_query_checks():
    import torch

    import pydiskann_b200 as dg

    ix = object.__new__(dg._Index)
    ix._X = np.zeros((1, 4), np.float32)
    s = SPFresh(4, device=None)
    s._h = object()
    try:
        for call in (lambda q: ix._params(q, 10, 32, 0, 0, None, None, None, None, False),
                     lambda q: s.search_arrays(q, 10, 4)):
            with pytest.raises(ValueError, match="^Query dim 3 != index dim 4$"):
                call(_AsCuda(torch.zeros(3)))
            with pytest.raises(ValueError, match="^Query dim 3 != index dim 4$"):
                call(_AsCuda(torch.zeros((2, 3))))
            with pytest.raises(ValueError, match="2-D batch"):
                call(_AsCuda(torch.zeros((2, 2, 4))))
            with pytest.raises(ValueError, match="must be float32"):
                call(_AsCuda(torch.zeros((2, 4), dtype=torch.float64)))
    finally:
        s._h = None


def test_autotune_reports_every_axis(monkeypatch):
    """Index.autotune passes the search to dg_index_autotune and returns the
    schedule dg_index_tuned_schedule reports: table bits, query order, CTAs
    per SM and warps per CTA, with the per-table timings that fitted."""
    import ctypes as C

    import pydiskann_b200 as dg

    class FakeLib:
        def dg_index_autotune(self, h, p, q, nq, reps, best, ms):
            assert nq == 3 and reps == 2
            arr = C.cast(ms, C.POINTER(C.c_float))
            for i in range(6):
                arr[i] = -1.0 if i == 5 else 1.0 + i
            best._obj.value = 10
            return 0

        def dg_index_tuned_schedule(self, h, hb, order, occ, wpb):
            hb._obj.value, order._obj.value, occ._obj.value, wpb._obj.value = 10, 1, 75, 2
            return 0

    monkeypatch.setattr(dg, "lib", lambda: FakeLib())
    ix = object.__new__(dg._Index)
    ix._X = np.zeros((1, 4), np.float32)
    ix._h = object()  # stands in for the device index
    try:
        t = ix.autotune(np.zeros((3, 4), np.float32), 10, 32, reps=2)
    finally:
        ix._h = None
    assert t == {"hbits": 10, "order": 1, "occ_pct": 75, "warps_per_cta": 2,
                 "ms": {8: 1.0, 9: 2.0, 10: 3.0, 11: 4.0, 12: 5.0}}
