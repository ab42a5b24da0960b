"""dg_search_batch_static: the search entry point for callers that cannot have
device memory allocated for them (a host whose device memory belongs to its
own pool manager, a latency-critical thread that must not pay cudaMalloc's
implicit synchronisation).  Its scratch lives in a fixed device array inside
libdgann; these checks call it through the C ABI and compare it with the
allocating dg_search_batch on the same inputs, twice in a row (the array
keeps the previous call's contents, so the second call shows it is reset).

Kept in a file of its own that runs last; it builds everything it needs, so
it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_search(index, Qd, k, L, traversal, rerank=0, filt=None, beams=None, sync=True):
    import torch

    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib

    nq = Qd.shape[0]
    ids = torch.empty((nq, k), dtype=torch.int32, device=Qd.device)
    ds = torch.empty((nq, k), dtype=torch.float32, device=Qd.device)
    cnt = torch.empty((nq,), dtype=torch.int32, device=Qd.device)
    p = _lib.SearchParams()
    p.k, p.beam_width, p.rerank_size, p.traversal = k, L, rerank, traversal
    p.flags = _lib.FLAG_DEVICE_PTRS | _lib.FLAG_STREAM
    p.stream = torch.cuda.current_stream(Qd.device).cuda_stream
    keep = []
    if filt is not None:
        arr, offs, pool, plen = dg._pack_programs([filt.program()])
        keep += [arr, pool]
        p.filter_ops, p.filter_nops = C.cast(arr, C.c_void_p), int(offs[-1])
        p.filter_pool, p.filter_pool_len = _lib.ptr(pool), plen
    if beams is not None:
        b = np.ascontiguousarray(beams, dtype=np.uint32)
        keep.append(b)
        p.per_query_beam = _lib.ptr(b)
    st = _lib.lib().dg_search_batch_static(index._h, C.byref(p), _lib.ptr(Qd), nq, _lib.ptr(ids), _lib.ptr(ds),
                                           _lib.ptr(cnt))
    if not sync:
        return st, (ids, ds, cnt)
    torch.cuda.synchronize()
    return st, ids.cpu().numpy().view(np.uint32), ds.cpu().numpy(), cnt.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def setup():
    import torch

    import pydiskann_b200 as dg
    from pydiskann_b200 import synth

    X = synth.mixture(3000, 128, 16, seed=31)
    Q = synth.mixture(150, 128, 16, seed=31, stream=synth.STREAM_QUERY)
    adj, med = dg.build_graph(X, 32, 64, 1.2, seed=4)
    labels = np.stack([np.arange(len(X)) % 4, np.arange(len(X)) % 9], 1).astype(np.uint64)
    idx = dg.FilteredDiskANN(X, adj, med, labels)
    idx.enable_bf16()
    Qd = torch.from_numpy(Q).cuda()
    # code traversals: int8 and PQ codes with an FP32 rerank
    q8 = dg.QuantizedDiskANN(X, adj, med)
    q8.attach_int8(*dg.int8_params(X))
    qpq = dg.QuantizedDiskANN(X, adj, med)
    qpq.attach_pq(dg.pq_train(X, 16, 256, 4, 3000, seed=5))
    # a base + delta shaped index: two entry points and tombstoned rows
    tomb = dg.DiskANN.from_graph(X, adj, med)
    dead = np.arange(7, len(X), 11, dtype=np.uint32)
    _lib_check(tomb, "dg_index_set_tombstones", dead, len(dead), 1, len(dead))
    _lib_check(tomb, "dg_index_set_entry_points", np.array([med, (med + 1234) % len(X)], dtype=np.uint32), 2)
    yield dg, {"main": idx, "int8": q8, "pq": qpq, "tomb": tomb}, Q, Qd
    for ix in (idx, q8, qpq, tomb):
        ix.close()


def _lib_check(index, name, arr, *args):
    from pydiskann_b200 import _lib

    st = getattr(_lib.lib(), name)(index._h, _lib.ptr(arr), *args)
    assert st == _lib.DG_OK, _lib.lib().dg_last_error()


@pytest.mark.parametrize("case", ["fp32", "bf16_rerank", "filtered", "uneven_beams", "int8_rerank",
                                  "pq_rerank", "tombstones_two_seeds"])
def test_static_matches_allocating_entry_point(setup, case):
    dg, ixs, Q, Qd = setup
    from pydiskann_b200 import _lib

    idx = {"int8_rerank": ixs["int8"], "pq_rerank": ixs["pq"], "tombstones_two_seeds": ixs["tomb"]}.get(case,
                                                                                                    ixs["main"])
    trav = {"bf16_rerank": _lib.TRAVERSE_BF16, "int8_rerank": _lib.TRAVERSE_CODES,
            "pq_rerank": _lib.TRAVERSE_CODES}.get(case, _lib.TRAVERSE_F32)
    rerank = 48 if case in ("bf16_rerank", "int8_rerank", "pq_rerank") else 0
    filt = dg.Filter.or_([dg.Filter.eq(0, 1), dg.Filter.range(1, 2, 4)]) if case == "filtered" else None
    beams = np.random.default_rng(3).integers(4, 120, size=len(Q)) if case == "uneven_beams" else None
    want = idx.search_arrays(Q, 10, 48, traversal=trav, rerank_size=rerank, filters=filt, per_query_beam=beams)
    for _ in range(2):  # the second call sees the previous call's scratch contents
        st, ids, ds, cnt = _static_search(idx, Qd, 10, 48, trav, rerank, filt, beams)
        assert st == _lib.DG_OK, _lib.lib().dg_last_error()
        assert np.array_equal(cnt, want[2])
        assert np.array_equal(ids, want[0])
        assert np.array_equal(ds, want[1])  # same kernel, same inputs: bit-identical


def test_static_rejects_parameters_beyond_its_array(setup):
    dg, ixs, Q, Qd = setup
    idx = ixs["main"]
    from pydiskann_b200 import _lib

    import torch

    big = torch.from_numpy(np.tile(Q, (500, 1))).cuda()  # 75k queries with per-query beams
    beams = np.full(big.shape[0], 32, dtype=np.uint32)
    st, _, _, _ = _static_search(idx, big, 10, 32, _lib.TRAVERSE_F32, beams=beams)
    assert st == _lib.DG_EINVAL
    assert b"static scratch" in _lib.lib().dg_last_error()


def test_updates_and_destroy_wait_for_a_static_search():
    """A static search still running on its own stream when the caller
    tombstones rows, rewrites rows and destroys the index (no synchronisation
    in between) returns the results of the index as it was: every update and
    the destroy wait for the search's completion event."""
    import torch

    import oracle
    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib, synth

    X = synth.mixture(6000, 128, 16, seed=41)
    Q = synth.mixture(3000, 128, 16, seed=41, stream=synth.STREAM_QUERY)
    adj, med = dg.build_graph(X, 32, 64, 1.2, seed=6)
    want = oracle.OracleIndex(X, adj, med).search(Q, 10, 200)
    idx = dg.DiskANN.from_graph(X, adj, med)
    Qd = torch.from_numpy(Q).cuda()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        st, (ids, ds, cnt) = _static_search(idx, Qd, 10, 200, _lib.TRAVERSE_F32, sync=False)
    assert st == _lib.DG_OK, _lib.lib().dg_last_error()
    # the nearest results of every query: tombstoned, then moved far away
    hit = np.unique(want[0][:, :3]).astype(np.uint32)
    _lib_check(idx, "dg_index_set_tombstones", hit, len(hit), 1, len(hit))
    far = np.full((1, X.shape[1]), 1e6, dtype=np.float32)
    for r in hit[:50]:
        assert _lib.lib().dg_index_update_rows(idx._h, int(r), 1, _lib.ptr(far), None, None) == _lib.DG_OK
    idx.close()
    torch.cuda.synchronize()
    assert np.array_equal(cnt.cpu().numpy().view(np.uint32), want[2])
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), want[0])
    assert np.array_equal(ds.cpu().numpy(), want[1])
