"""Server.run_trace's request records, up to the library call (no GPU).

run_trace packs every request's filter program into shared arrays and points
each DgRequest into them.  A stand-in dg_server_run_trace reads the records
back through those pointers: each request must carry its own k / beam /
rerank / traversal and exactly its own postfix program, with IN offsets
relative to its own value pool, and the per-request results must come back
sliced by their k.
"""
import ctypes as C

import numpy as np
import pytest

import pydiskann_b200.serve as serve_mod
from pydiskann_b200 import Filter, _lib
from pydiskann_b200.serve import _REQ_DTYPE, Server

OP_DTYPE = np.dtype({"names": ["op", "field", "a", "b"], "formats": [np.uint32, np.uint32, np.uint64, np.uint64],
                     "offsets": [0, 4, 8, 16], "itemsize": C.sizeof(_lib.FilterOp)})


def _arr(p, dtype, n):
    return np.frombuffer((C.c_char * (n * np.dtype(dtype).itemsize)).from_address(int(p)), dtype=dtype).copy()


class FakeServeLib:
    def __init__(self):
        self.requests = None

    def dg_server_create(self, ih, cfg, out):
        out._obj.value = 1
        return 0

    def dg_server_destroy(self, h):
        return 0

    def dg_server_run_trace(self, h, q, n, reqs, arrival, timeout, ids, ds, cnt, lat, wall):
        R = _arr(reqs.value, _REQ_DTYPE, n)
        progs = []
        for r in R:
            ops = _arr(r["ops"], OP_DTYPE, r["nops"]).tolist() if r["nops"] else []
            pool = _arr(r["pool"], np.uint64, r["npool"]).tolist() if r["npool"] else []
            progs.append(([tuple(int(x) for x in o) for o in ops], [int(v) for v in pool]))
        self.requests = (R, progs)
        ks = R["k"].astype(np.int64)
        total = int(ks.sum())
        out_ids = np.ctypeslib.as_array(C.cast(ids, C.POINTER(C.c_uint32)), (total,))
        out_cnt = np.ctypeslib.as_array(C.cast(cnt, C.POINTER(C.c_uint32)), (n,))
        out_lat = np.ctypeslib.as_array(C.cast(lat, C.POINTER(C.c_double)), (n,))
        off = 0
        for i in range(n):  # request i answers ids 100 i + j, for min(k, 3) results
            c = min(int(ks[i]), 3)
            out_ids[off:off + c] = 100 * i + np.arange(c)
            out_cnt[i] = c
            out_lat[i] = float(i)
            off += int(ks[i])
        wall._obj.value = 7.0
        return 0


class _Idx:
    dim, _h = 4, None


@pytest.fixture()
def srv(monkeypatch):
    fake = FakeServeLib()
    monkeypatch.setattr(serve_mod, "lib", lambda: fake)
    s = Server(_Idx())
    yield s, fake
    s._h = None


def test_per_request_programs_and_results(srv):
    s, fake = srv
    filters = [Filter.eq(0, 3), None, Filter.in_(1, [9, 4, 7]), Filter.none(),
               Filter.and_([Filter.in_(0, [1, 2]), Filter.or_([Filter.lt(1, 5), Filter.in_(2, [8])])]),
               Filter.range(2, 10, 20)]
    n = len(filters)
    ks = np.array([1, 5, 2, 4, 3, 10], np.uint32)
    out = s.run_trace(np.zeros((n, 4), np.float32), np.arange(n) * 10.0, k=ks, beam_width=32, rerank_size=8,
                      traversal="bf16", filters=filters)
    R, progs = fake.requests
    assert R["k"].tolist() == ks.tolist() and set(R["beam"]) == {32} and set(R["rerank"]) == {8}
    assert set(R["trav"]) == {_lib.TRAVERSE_BF16}
    for f, (ops, pool) in zip(filters, progs):
        want = ([], []) if f is None or f.is_none() else f.program()
        assert (ops, pool) == (list(want[0]), list(want[1])), f
    for i in range(n):
        c = min(int(ks[i]), 3)
        assert out["ids"][i].tolist() == [100 * i + j for j in range(c)] and len(out["dists"][i]) == c
    assert out["latency_us"].tolist() == list(range(n)) and out["wall_us"] == 7.0


def test_trace_validation(srv):
    s, _ = srv
    with pytest.raises(ValueError, match="one arrival time per query"):
        s.run_trace(np.zeros((3, 4), np.float32), np.zeros(2))
    with pytest.raises(ValueError, match="one filter per query"):
        s.run_trace(np.zeros((3, 4), np.float32), np.zeros(3), filters=[Filter.eq(0, 1)] * 2)
    with pytest.raises(ValueError, match="Query dim 3 != index dim 4"):
        s.run_trace(np.zeros((3, 3), np.float32), np.zeros(3))
