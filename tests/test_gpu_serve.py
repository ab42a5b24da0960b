"""Continuous-batching serving loop (dg_server_*).

The property checked is the one a serving loop must keep: every request's
result is the same when it is served alone and when it is batched with other
requests of different beams, traversals, rerank sizes and filters that arrive
while earlier batches are on the GPU.  Tolerance: none (ids, counts and
distances bit-identical).  The FP32 requests are also checked against the
oracle's restatement of DiskANN::search_with_dists (src/lib.rs:683-714).
"""
import numpy as np
import pytest

import pydiskann_b200 as dg
from pydiskann_b200 import _lib

pytestmark = pytest.mark.gpu

FILTERS = [
    dg.Filter.eq(0, 3),
    dg.Filter.range(1, 10, 40),
    dg.Filter.or_([dg.Filter.eq(2, 6), dg.Filter.in_(1, [1, 2, 3, 99])]),
]


def _labels(n, seed=2):
    rng = np.random.default_rng(seed)
    return np.stack([np.arange(n) % 5, rng.integers(0, 100, n), rng.integers(0, 7, n)], 1).astype(np.uint64)


@pytest.fixture(scope="module")
def qindex(small_data, small_graph):
    X, _ = small_data
    adj, med = small_graph
    s, off = dg.int8_params(X)
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_int8(s, off)
    q.attach_labels(_labels(len(X)))
    q.enable_bf16()
    yield q
    q.close()


def _mix(n, seed=5):
    rng = np.random.default_rng(seed)
    k = rng.choice([5, 10, 20], n)
    L = rng.choice([16, 24, 40, 64, 100], n)
    trav = rng.choice([_lib.TRAVERSE_F32, _lib.TRAVERSE_BF16, _lib.TRAVERSE_CODES], n)
    rerank = np.where(trav == _lib.TRAVERSE_CODES, rng.choice([0, 30], n), 0)
    filt = [FILTERS[rng.integers(len(FILTERS))] if rng.random() < 0.25 else None for _ in range(n)]
    return k, L, trav, rerank, filt


def _alone(index, q, k, L, trav, rr, f):
    ids, ds, cnt = index.search_arrays(q.reshape(1, -1), int(k), int(L), traversal=int(trav), rerank_size=int(rr),
                                       filters=f)
    return ids[0, : cnt[0]], ds[0, : cnt[0]]


def test_same_alone_and_in_the_mix(qindex, small_data, oracle, small_graph):
    X, Q = small_data
    n = 600
    Qn = Q[np.arange(n) % len(Q)]
    k, L, trav, rr, filt = _mix(n)
    arrivals = dg.poisson_arrivals(n, 50_000, seed=1)
    with dg.Server(qindex, max_batch=64, streams=4, max_k=32, max_wait_us=100) as srv:
        out = srv.run_trace(Qn, arrivals, k=k, beam_width=L, rerank_size=rr, traversal=trav, filters=filt)
        st = srv.stats()
    assert st["served"] == n
    assert st["batches"] < n  # requests were batched
    assert (out["latency_us"] > 0).all()
    for i in range(n):
        ai, ad = _alone(qindex, Qn[i], k[i], L[i], trav[i], rr[i], filt[i])
        assert np.array_equal(out["ids"][i], ai), i
        assert np.array_equal(out["dists"][i], ad), i
    # the FP32 unfiltered requests against the oracle
    adj, med = small_graph
    o = oracle.OracleIndex(X, adj, med)
    for i in np.nonzero((trav == _lib.TRAVERSE_F32) & np.array([f is None for f in filt]))[0][:80]:
        oi, od, oc = o.search(Qn[i:i + 1], int(k[i]), int(L[i]))
        assert np.array_equal(out["ids"][i], oi[0, : oc[0]]), i
        assert np.array_equal(out["dists"][i], od[0, : oc[0]]), i


def test_overlapping_batches_and_submit_wait(qindex, small_data):
    """A burst larger than one batch keeps several batches in flight; tickets
    submitted one by one return what the single search returns."""
    _, Q = small_data
    with dg.Server(qindex, max_batch=16, streams=4, max_k=16) as srv:
        tickets = [srv.submit(Q[i], k=10, beam_width=64, traversal="f32") for i in range(len(Q))]
        res = [srv.wait(t, timeout=30) for t in tickets]
        st = srv.stats()
    assert st["served"] == len(Q) and st["max_in_flight"] >= 2
    ids, ds, cnt = qindex.search_arrays(Q, 10, 64, traversal=_lib.TRAVERSE_F32)
    for i, (ri, rd, lat) in enumerate(res):
        assert np.array_equal(ri, ids[i, : cnt[i]]) and np.array_equal(rd, ds[i, : cnt[i]]) and lat > 0


def test_mixed_k_in_one_launch(qindex, small_data):
    """One batched call carries a k per query (k in {10, 100}, with and
    without filters): every row equals the query's own search with its k."""
    _, Q = small_data
    n = 96
    k = np.where(np.arange(n) % 2 == 0, 10, 100).astype(np.uint32)
    filt = [FILTERS[i % 3] if i % 4 == 1 else dg.Filter.none() for i in range(n)]
    ids, ds, cnt = qindex.search_arrays(Q[:n], 100, 64, traversal=_lib.TRAVERSE_BF16, filters=filt, per_query_k=k)
    for i in range(n):
        ai, ad = _alone(qindex, Q[i], k[i], 64, _lib.TRAVERSE_BF16, 0, None if filt[i].is_none() else filt[i])
        assert cnt[i] == len(ai) <= k[i]
        assert np.array_equal(ids[i, : cnt[i]], ai) and np.array_equal(ds[i, : cnt[i]], ad), i
        assert (ids[i, cnt[i]:] == _lib.PAD).all() and np.isinf(ds[i, cnt[i]:]).all()
    with pytest.raises(ValueError):
        qindex.search_arrays(Q[:4], 10, 64, per_query_k=np.array([5, 11, 3, 2]))


def test_serving_mixes_k_and_admits_by_memory(qindex, small_data):
    """A burst of requests with k in {10, 100}: batches mix k (fewer batches
    than one class per k would need), and under a budget that holds only a few
    requests at once the dispatcher trims batches to what fits and waits for
    memory; every result is the request's own search."""
    _, Q = small_data
    n = 256
    Qn = Q[np.arange(n) % len(Q)]
    k = np.where(np.arange(n) % 2 == 0, 10, 100)
    with dg.Server(qindex, max_batch=64, streams=2, max_k=100) as srv:
        out = srv.run_trace(Qn, np.zeros(n), k=k, beam_width=48, traversal=_lib.TRAVERSE_F32)
        roomy = srv.stats()
    per_request = 512 + 1024 + 256 + 256  # query, results at k = 100, beam, k (256-byte parts)
    with dg.Server(qindex, max_batch=64, streams=2, max_k=100, hbm_budget_bytes=6 * per_request) as srv:
        tight = srv.run_trace(Qn, np.zeros(n), k=k, beam_width=48, traversal=_lib.TRAVERSE_F32)
        st = srv.stats()
    assert roomy["served"] == st["served"] == n
    assert roomy["batches"] <= n // 64 + 2  # k = 10 and k = 100 share launches
    assert st["batches"] > roomy["batches"]  # trimmed to the budget
    for res in (out, tight):
        for i in range(n):
            ai, ad = _alone(qindex, Qn[i], k[i], 48, _lib.TRAVERSE_F32, 0, None)
            assert np.array_equal(res["ids"][i], ai) and np.array_equal(res["dists"][i], ad), i


def test_server_errors(qindex, small_data):
    _, Q = small_data
    with pytest.raises(dg.DgError) as e:  # one request at max_k does not fit the budget
        dg.Server(qindex, max_batch=1024, streams=4, max_k=100, hbm_budget_bytes=1024)
    assert e.value.status == _lib.DG_ENOMEM
    with dg.Server(qindex, max_batch=8, streams=1, max_k=10, max_wait_us=300_000) as srv:
        with pytest.raises(ValueError):
            srv.submit(Q[0], k=11)
        with pytest.raises(ValueError):
            srv.submit(Q[0][:5])
        t = srv.submit(Q[0], k=5, beam_width=32, traversal="f32")
        # a partial batch waits up to 300 ms to fill: a 10 ms wait expires and
        # leaves the ticket pending
        with pytest.raises(dg.DgError) as e:
            srv.wait(t, timeout=0.01)
        assert e.value.status == _lib.DG_ETIMEOUT
        ids, ds, _ = srv.wait(t, timeout=10)
        ai, ad = _alone(qindex, Q[0], 5, 32, _lib.TRAVERSE_F32, 0, None)
        assert np.array_equal(ids, ai) and np.array_equal(ds, ad)
