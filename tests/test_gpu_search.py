"""GPU beam search vs the CPU oracle, through the C ABI.

The seeded data is integer valued, so every FP32 (and BF16 / F16) distance is
exact in any summation order: ids, counts and distances must be bit-identical
to the oracle's.  Non-integer data (cosine) is compared within 1e-5 relative.
"""
import numpy as np
import pytest

import pydiskann_b200 as dg
from pydiskann_b200 import _lib

pytestmark = pytest.mark.gpu


def assert_same(g, o):
    gi, gd, gc = g
    oi, od, oc = o
    assert (np.asarray(gc) == oc).all(), np.nonzero(np.asarray(gc) != oc)
    bad = np.nonzero((np.asarray(gi) != oi).any(1))[0]
    assert len(bad) == 0, (bad[:5], np.asarray(gi)[bad[:2]], oi[bad[:2]])
    assert np.array_equal(np.asarray(gd), od)


@pytest.fixture(scope="module")
def gindex(small_data, small_graph):
    X, _ = small_data
    adj, med = small_graph
    idx = dg.DiskANN.from_graph(X, adj, med)
    yield idx
    idx.close()


@pytest.fixture(scope="module")
def oindex(oracle, small_data, small_graph):
    X, _ = small_data
    adj, med = small_graph
    return oracle.OracleIndex(X, adj, med)


@pytest.mark.parametrize("L", [1, 16, 64, 200, 700])
@pytest.mark.parametrize("k", [1, 10])
def test_fp32_matches_oracle(gindex, oindex, small_data, L, k):
    _, Q = small_data
    assert_same(gindex.search_arrays(Q, k, L), oindex.search(Q, k, L))


def test_bf16_traversal_matches_oracle(gindex, oindex, small_data):
    """Integer data is exact in BF16: the BF16 traversal equals the FP32 one, and
    the FP32 rerank of its whole working set returns the same distances."""
    _, Q = small_data
    gindex.enable_bf16()
    assert_same(gindex.search_arrays(Q, 10, 64, traversal=_lib.TRAVERSE_BF16), oindex.search(Q, 10, 64))
    assert_same(gindex.search_arrays(Q, 10, 64, traversal=_lib.TRAVERSE_BF16, rerank_size=64),
                oindex.search(Q, 10, 64))


def test_stats_and_uneven_beams(gindex, oindex, small_data):
    _, Q = small_data
    L = np.random.default_rng(1).integers(8, 257, size=len(Q)).astype(np.uint32)
    gi, gd, gc, st = gindex.search_arrays(Q, 10, 64, per_query_beam=L, with_stats=True)
    oi, od, oc, ost = oindex.search(Q, 10, 64, per_query_L=L, with_stats=True)
    assert_same((gi, gd, gc), (oi, od, oc))
    assert (st[:, 0] == ost[:, 0]).all()  # same number of expansions
    assert (st[:, 1] >= ost[:, 1]).all()  # forgotten visits are re-evaluated, never skipped


def test_device_pointer_path(gindex, oindex, small_data):
    import torch

    _, Q = small_data
    Qd = torch.from_numpy(Q).cuda()
    ids, ds, cnt = gindex.search_arrays(Qd, 10, 64)
    torch.cuda.synchronize()
    oi, od, oc = oindex.search(Q, 10, 64)
    assert_same((ids.cpu().numpy().view(np.uint32), ds.cpu().numpy(), cnt.cpu().numpy().view(np.uint32)),
                (oi, od, oc))


def test_pq_codes_and_search_match_oracle(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    cb = dg.pq_train(X, num_subspaces=16, num_centroids=256, kmeans_iterations=8, training_sample_size=3000, seed=4)
    codes = oracle.pq_encode(X, cb)
    assert np.array_equal(dg.pq_encode(X, cb), codes)
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_pq(cb)  # encodes on the GPU
    o = oracle.OracleIndex(X, adj, med)
    o.set_pq(cb, codes)
    for L, rr in ((32, 0), (64, 64), (128, 20)):
        assert_same(q.search_arrays(Q, 10, L, rerank_size=rr), o.search(Q, 10, L, rerank=rr, use_codes=True))
    q.close()


@pytest.mark.parametrize("sample,iters", [(2500, 4), (0, 3)])
def test_pq_training_matches_oracle(oracle, small_data, sample, iters):
    """The GPU k-means (sample, k-means++ seeding, Lloyd steps with f64 centre
    sums) equals the oracle's restatement of ProductQuantizer::train
    (src/pq.rs:290-410) from the same seed, codebooks bit for bit on
    integer-valued data (every sum is exact)."""
    X, _ = small_data
    got = dg.pq_train(X, num_subspaces=16, num_centroids=256, kmeans_iterations=iters,
                      training_sample_size=sample, seed=4)
    want = oracle.pq_train(X, 16, 256, iters, sample, 4)
    assert np.array_equal(got, want), np.argwhere(got != want)[:5]


def test_int8_codes_and_search_match_oracle(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    s, off = dg.int8_params(X)
    assert (s, off) == oracle.int8_train(X)
    codes = oracle.int8_encode(X, s, off)
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_int8(s, off)
    o = oracle.OracleIndex(X, adj, med)
    o.set_int8(s, off, codes)
    for L, rr in ((48, 0), (64, 32)):
        assert_same(q.search_arrays(Q, 10, L, rerank_size=rr), o.search(Q, 10, L, rerank=rr, use_codes=True))
    q.close()


def test_f16_search_matches_oracle(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_f16()
    o = oracle.OracleIndex(X, adj, med)
    o.set_f16(oracle.f16_encode(X))
    assert_same(q.search_arrays(Q, 10, 64), o.search(Q, 10, 64, use_codes=True))
    q.close()


def test_rabitq_codes_and_search_match_oracle(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    cen, signs = dg.rabitq_params(X, seed=3)
    P = dg.rabitq_padded(X.shape[1])
    codes = oracle.rabitq_encode(X, P, cen, signs)
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_rabitq(cen, signs)
    o = oracle.OracleIndex(X, adj, med)
    o.set_rabitq(P, cen, signs, codes)
    for L, rr in ((64, 0), (64, 64)):
        assert_same(q.search_arrays(Q, 10, L, rerank_size=rr), o.search(Q, 10, L, rerank=rr, use_codes=True))
    q.close()


def _labels(n, seed=2):
    rng = np.random.default_rng(seed)
    return np.stack([np.arange(n) % 5, rng.integers(0, 100, n), rng.integers(0, 7, n)], 1).astype(np.uint64)


FILTERS = [
    dg.Filter.eq(0, 3),
    dg.Filter.range(1, 10, 30),
    dg.Filter.and_([dg.Filter.eq(0, 1), dg.Filter.gt(1, 50)]),
    dg.Filter.or_([dg.Filter.eq(2, 6), dg.Filter.in_(1, [1, 2, 3, 99])]),
    dg.Filter.lt(1, 2),
]


@pytest.mark.parametrize("fi", range(len(FILTERS)))
def test_filtered_matches_oracle(oracle, small_data, small_graph, fi):
    X, Q = small_data
    adj, med = small_graph
    lab = _labels(len(X))
    f = FILTERS[fi]
    g = dg.FilteredDiskANN(X, adj, med, lab)
    o = oracle.OracleIndex(X, adj, med)
    o.set_labels(lab)
    ops, pool = f.program()
    for k, L in ((10, 32), (10, 64), (5, 16)):
        assert_same(g.search_arrays(Q, k, L, filters=f), o.search(Q, k, L, filter_ops=ops, filter_pool=pool))
    assert g.count_matching(f) == sum(f.matches(list(map(int, r))) for r in lab)
    g.close()


def test_per_query_filters_match_oracle(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    lab = _labels(len(X))
    g = dg.FilteredDiskANN(X, adj, med, lab)
    o = oracle.OracleIndex(X, adj, med)
    o.set_labels(lab)
    fl = [FILTERS[i % len(FILTERS)] if i % 7 else dg.Filter.none() for i in range(len(Q))]
    gi, gd, gc = g.search_arrays(Q, 10, 40, filters=fl)
    for i, f in enumerate(fl):
        ops, pool = f.program()
        oi, od, oc = o.search(Q[i:i + 1], 10, 40, filter_ops=ops or None, filter_pool=pool)
        assert gc[i] == oc[0] and (gi[i] == oi[0]).all() and np.array_equal(gd[i], od[0]), i
    g.close()


def test_quantized_filtered_matches_oracle(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    lab = _labels(len(X))
    s, off = dg.int8_params(X)
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_int8(s, off)
    q.attach_labels(lab)
    o = oracle.OracleIndex(X, adj, med)
    o.set_int8(s, off, oracle.int8_encode(X, s, off))
    o.set_labels(lab)
    f = FILTERS[3]
    ops, pool = f.program()
    assert_same(q.search_arrays(Q, 10, 32, rerank_size=16, filters=f),
                o.search(Q, 10, 32, rerank=16, use_codes=True, filter_ops=ops, filter_pool=pool))
    q.close()


def test_cosine_within_tolerance(oracle):
    from pydiskann_b200 import synth

    X, Q = synth.cosine(3000, 50, 96, seed=5)
    adj, med = oracle.build_vamana(X, 24, 48, 1.2, seed=3, metric=oracle.COSINE)
    g = dg.DiskANN.from_graph(X, adj, med, metric="cosine")
    o = oracle.OracleIndex(X, adj, med, oracle.COSINE)
    gi, gd, gc = g.search_arrays(Q, 10, 64)
    oi, od, oc = o.search(Q, 10, 64)
    same = np.mean([len(set(gi[i]) & set(oi[i])) / 10 for i in range(len(Q))])
    assert same >= 0.98
    for i in range(len(Q)):
        for j in range(10):
            if gi[i, j] == oi[i, j]:
                assert abs(gd[i, j] - od[i, j]) <= 1e-5 * max(1e-3, abs(od[i, j])) + 1e-6
    g.close()


def test_edge_cases():
    X = np.array([[1.0, 2.0, 3.0]], dtype=np.float32)
    idx = dg.DiskANN.build(X)
    assert idx.search([1.0, 2.0, 3.0], 1, 8) == [0]
    assert idx.search([0.0, 0.0, 0.0], 10, 8) == [0]
    with pytest.raises(ValueError):
        idx.search([1.0, 2.0], 1, 8)
    with pytest.raises(RuntimeError):
        dg.DiskANN.build(np.zeros((0, 4), dtype=np.float32))
    with pytest.raises(ValueError):
        dg.DiskANN.build(X, metric="manhattan")
    Y = np.tile(np.array([[1.0, 2.0, 3.0]], dtype=np.float32), (10, 1))
    r = dg.DiskANN.build(Y).search_with_dists([1.0, 2.0, 3.0], 5, 8)
    assert len(r) == 5 and all(d < 1e-6 for _, d in r)
    rng = np.random.default_rng(201)
    Z = rng.random((50, 16), dtype=np.float32)
    r = dg.DiskANN.build(Z).search_with_dists(Z[0], 1, 1)
    assert len(r) == 1 and r[0][1] >= 0.0


# Cosine / dot over PQ, RaBitQ and int8 codes: the reference decodes the code
# and evaluates the metric (src/quantized.rs:28-36, src/pq.rs:151-160,
# src/rabitq.rs:224-238, src/sq.rs:222-225).  The kernel takes
# q . decode(code) from a query-centroid inner-product table (PQ), in the
# rotated space (RaBitQ), or as s (q . c) + o sum(q) with q . c on the tensor
# cores (int8, the query as four 8-bit digit columns), so the sum is grouped
# differently from the decoded vector's sequential sum.  Tolerance: ids agree
# with the oracle except among near-ties (>= 98 % overlap), distances of common
# ids within 1e-5 relative + 2e-6 absolute.
DECODE_CASES = [("pq", "cosine", 96), ("pq", "dot", 64), ("rabitq", "cosine", 96), ("rabitq", "dot", 64),
                ("rabitq", "cosine", 128), ("int8", "cosine", 96), ("int8", "dot", 64), ("int8", "cosine", 768),
                ("int8", "dot", 200)]


@pytest.mark.parametrize("quant,metric,d", DECODE_CASES)
def test_decoded_metrics_within_tolerance(oracle, quant, metric, d):
    from pydiskann_b200 import synth

    X, Q = synth.cosine(3000, 60, d, seed=6)
    om = oracle.COSINE if metric == "cosine" else oracle.DOT
    adj, med = oracle.build_vamana(X, 24, 48, 1.2, seed=3, metric=om)
    q = dg.QuantizedDiskANN(X, adj, med, metric=metric)
    o = oracle.OracleIndex(X, adj, med, om)
    if quant == "pq":
        cb = dg.pq_train(X, 8, 64, 10, 3000, seed=1)
        q.attach_pq(cb)
        o.set_pq(cb, oracle.pq_encode(X, cb))
    elif quant == "int8":
        s, off = dg.int8_params(X)
        q.attach_int8(s, off)
        o.set_int8(s, off, oracle.int8_encode(X, s, off))
    else:
        cen, signs = dg.rabitq_params(X, seed=3)
        P = dg.rabitq_padded(d)
        q.attach_rabitq(cen, signs)
        o.set_rabitq(P, cen, signs, oracle.rabitq_encode(X, P, cen, signs))
    for rr in (0, 32):
        gi, gd, gc = q.search_arrays(Q, 10, 48, rerank_size=rr)
        oi, od, oc = o.search(Q, 10, 48, rerank=rr, use_codes=True)
        assert np.array_equal(gc, oc)
        same = np.mean([len(set(gi[i]) & set(oi[i])) / 10 for i in range(len(Q))])
        assert same >= 0.98, (quant, metric, rr, same)
        m = gi == oi
        assert np.all(np.abs(gd[m] - od[m]) <= 1e-5 * np.abs(od[m]) + 2e-6), (quant, metric, rr)
    q.close()


def test_host_pipeline_matches_device_call(small_data, small_graph):
    """Host-pointer calls of >= 4096 queries run as a pipeline of chunks over
    several streams; results, counts and stats equal the single device-pointer
    launch, with per-query beams and per-query filter programs."""
    import torch

    from pydiskann_b200 import synth

    X, _ = small_data
    adj, med = small_graph
    g = dg.FilteredDiskANN(X, adj, med, _labels(len(X)))
    Q = synth.mixture(9000, 128, 32, seed=8, stream=synth.STREAM_QUERY)
    beams = (16 + np.arange(len(Q)) % 50).astype(np.uint32)
    fl = [FILTERS[i % len(FILTERS)] if i % 3 == 0 else dg.Filter.none() for i in range(len(Q))]
    for kw in ({}, {"per_query_beam": beams}, {"per_query_beam": beams, "filters": fl}):
        hi, hd, hc, hs = g.search_arrays(Q, 10, 40, with_stats=True, **kw)
        di, dd, dc, ds = g.search_arrays(torch.from_numpy(Q).cuda(), 10, 40, with_stats=True, **kw)
        torch.cuda.synchronize()
        assert np.array_equal(hc, dc.cpu().numpy().view(np.uint32))
        assert np.array_equal(hi, di.cpu().numpy().view(np.uint32))
        assert np.array_equal(hd, dd.cpu().numpy())
        assert np.array_equal(hs, ds.cpu().numpy().view(np.uint32))
    g.close()


def test_pinned_host_buffers(small_data, small_graph):
    """Pinned host buffers (torch pin_memory, as a serving host keeps them)
    give the results of pageable buffers and of the device call, for a single
    launch and for the chunk pipeline, with per-query beams and filters."""
    import torch

    from pydiskann_b200 import synth

    X, _ = small_data
    adj, med = small_graph
    g = dg.FilteredDiskANN(X, adj, med, _labels(len(X)))
    for nq in (300, 9000):
        Q = synth.mixture(nq, 128, 32, seed=9, stream=synth.STREAM_QUERY)
        beams = (16 + np.arange(nq) % 50).astype(np.uint32)
        fl = [FILTERS[i % len(FILTERS)] if i % 4 == 0 else dg.Filter.none() for i in range(nq)]
        Qp = torch.from_numpy(Q).pin_memory().numpy()
        for kw in ({}, {"per_query_beam": beams, "filters": fl}):
            out = (torch.zeros((nq, 10), dtype=torch.int32).pin_memory().numpy().view(np.uint32),
                   torch.zeros((nq, 10), dtype=torch.float32).pin_memory().numpy(),
                   torch.zeros((nq,), dtype=torch.int32).pin_memory().numpy().view(np.uint32))
            zi, zd, zc = g.search_arrays(Qp, 10, 40, out=out, **kw)
            assert zi is out[0]
            hi, hd, hc = g.search_arrays(Q, 10, 40, **kw)
            di, dd, dc = g.search_arrays(torch.from_numpy(Q).cuda(), 10, 40, **kw)
            torch.cuda.synchronize()
            assert np.array_equal(zc, hc) and np.array_equal(zi, hi) and np.array_equal(zd, hd)
            assert np.array_equal(zc, dc.cpu().numpy().view(np.uint32))
            assert np.array_equal(zi, di.cpu().numpy().view(np.uint32))
    g.close()


def test_autotune_keeps_results(oracle, small_data, small_graph):
    """dg_index_autotune tries every visited-table size, keeps the fastest, and
    searches afterwards return exactly what the oracle returns (a smaller table
    only recomputes distances of forgotten ids)."""
    X, Q = small_data
    adj, med = small_graph
    lab = _labels(len(X))
    s, off = dg.int8_params(X)
    q = dg.QuantizedDiskANN(X, adj, med)
    q.attach_int8(s, off)
    q.attach_labels(lab)
    o = oracle.OracleIndex(X, adj, med)
    o.set_int8(s, off, oracle.int8_encode(X, s, off))
    o.set_labels(lab)
    f = FILTERS[3]
    ops, pool = f.program()
    for kw, okw in (({}, {}), ({"filters": f}, {"filter_ops": ops, "filter_pool": pool})):
        t = q.autotune(Q, 10, 48, rerank_size=24, reps=2, **kw)
        assert 8 <= t["hbits"] <= 13 and t["hbits"] in t["ms"] and len(t["ms"]) >= 3
        assert_same(q.search_arrays(Q, 10, 48, rerank_size=24, **kw),
                    o.search(Q, 10, 48, rerank=24, use_codes=True, **okw))
    import os

    # every schedule axis at its extremes, forced: identical results, with
    # per-query beams and filters riding along with the reordered queries
    beams = np.random.default_rng(2).integers(8, 64, len(Q)).astype(np.uint32)
    filt = [FILTERS[i % len(FILTERS)] for i in range(len(Q))]
    want_b = o.search(Q, 10, 48, rerank=24, use_codes=True, per_query_L=beams)
    for env in ({"DG_HBITS": "8"}, {"DG_HBITS": "13"}, {"DG_ORDER": "1"}, {"DG_ORDER": "1", "DG_HBITS": "8"},
                {"DG_OCC_PCT": "50"}, {"DG_OCC_PCT": "75", "DG_ORDER": "1"}, {"DG_WPB": "1"},
                {"DG_WPB": "2", "DG_ORDER": "1", "DG_HBITS": "13"}):
        os.environ.update(env)
        try:
            assert_same(q.search_arrays(Q, 10, 48, rerank_size=24), o.search(Q, 10, 48, rerank=24, use_codes=True))
            assert_same(q.search_arrays(Q, 10, 48, rerank_size=24, per_query_beam=beams), want_b)
            got = q.search_arrays(Q, 10, 48, rerank_size=24, filters=filt)
            for i in range(0, len(Q), 7):
                fo, fp = filt[i].program()
                wi, wd, wc = o.search(Q[i:i + 1], 10, 48, rerank=24, use_codes=True, filter_ops=fo, filter_pool=fp)
                assert got[2][i] == wc[0] and np.array_equal(got[0][i], wi[0]) and np.array_equal(got[1][i], wd[0])
        finally:
            for k_ in env:
                del os.environ[k_]
    q.close()


def test_autotune_schedule_axes(oracle, small_data, small_graph):
    """The tuner's choice covers the four axes (table size, query order,
    CTAs per SM, warps per CTA) and a device-pointer search of 3000 queries after tuning --
    ordered or not -- returns the oracle's results."""
    import torch

    X, Q = small_data
    adj, med = small_graph
    ix = dg.DiskANN.from_graph(X, adj, med)
    ix.enable_bf16()
    Qb = np.concatenate([Q] * 15)
    t = ix.autotune(Qb, 10, 40, traversal=_lib.TRAVERSE_BF16, rerank_size=40, reps=2)
    assert 8 <= t["hbits"] <= 13 and t["order"] in (0, 1) and t["occ_pct"] in (50, 75, 100)
    assert t["warps_per_cta"] in (1, 2, 4)
    o = oracle.OracleIndex(X, adj, med)
    o.set_bf16()
    want = o.search(Qb, 10, 40, rerank=40, use_codes=True)
    got = ix.search_arrays(torch.from_numpy(Qb).cuda(), 10, 40, traversal=_lib.TRAVERSE_BF16, rerank_size=40)
    assert_same(tuple(g.cpu().numpy().view(np.uint32) if g.dtype != torch.float32 else g.cpu().numpy()
                      for g in got), want)
    ix.close()


@pytest.mark.parametrize("d", [48, 96, 200, 768])
def test_other_dims_match_oracle(oracle, d):
    """Dimensions that are not multiples of 128: padded rows (dpad = 32-multiple),
    ragged 16-byte chunk assignments in the int8 tensor-core tiles (d = 96, 200
    give 6 and 14 chunks over 4 lanes) and long rows (d = 768).  FP32, BF16 and
    int8 + rerank, bit-identical on integer data."""
    from pydiskann_b200 import synth

    X = synth.mixture(2500, d, 24, seed=30 + d)
    Q = synth.mixture(120, d, 24, seed=30 + d, stream=synth.STREAM_QUERY)
    if d * 255 * 255 >= 1 << 24:  # keep every FP32 partial sum an exact integer
        X, Q = np.floor(X / 2), np.floor(Q / 2)
    adj, med = oracle.build_vamana(X, 24, 48, 1.2, seed=4)
    o = oracle.OracleIndex(X, adj, med)
    g = dg.QuantizedDiskANN(X, adj, med)
    g.enable_bf16()
    s, off = dg.int8_params(X)
    g.attach_int8(s, off)
    assert_same(g.search_arrays(Q, 10, 40, traversal=_lib.TRAVERSE_F32), o.search(Q, 10, 40))
    # integer data is exact in BF16: the BF16 traversal (+ FP32 rerank) equals FP32
    assert_same(g.search_arrays(Q, 10, 40, traversal=_lib.TRAVERSE_BF16, rerank_size=40), o.search(Q, 10, 40))
    o.set_int8(s, off, oracle.int8_encode(X, s, off))
    for L, rr in ((24, 0), (40, 40)):
        assert_same(g.search_arrays(Q, 10, L, rerank_size=rr), o.search(Q, 10, L, rerank=rr, use_codes=True))
    g.close()


@pytest.mark.parametrize("metric", ["l2", "cosine"])
def test_fp8_traversal_within_tolerance(oracle, metric):
    """FP8 traversal (no counterpart in the reference): codes equal the oracle's
    restatement of e4m3 round-to-nearest-even with saturation bit for bit; the
    tensor cores accumulate e . q' in their own order, so traversal distances
    agree within 1e-5 (|q|^2 + |x|^2) and ids except near-ties; after the FP32
    rerank, distances of common ids are exact."""
    from pydiskann_b200 import synth

    if metric == "l2":
        X = synth.mixture(3000, 128, 24, seed=41)
        Q = synth.mixture(150, 128, 24, seed=41, stream=synth.STREAM_QUERY)
        om = oracle.L2SQ
    else:
        X, Q = synth.cosine(3000, 150, 96, seed=42)
        om = oracle.COSINE
    gc, gs = dg.fp8_encode(X)
    oc, osc = oracle.fp8_encode(X)
    assert np.array_equal(gc, oc) and np.array_equal(gs, osc)
    adj, med = oracle.build_vamana(X, 24, 48, 1.2, seed=5, metric=om)
    g = dg.DiskANN.from_graph(X, adj, med, metric=metric)
    g.enable_fp8()
    o = oracle.OracleIndex(X, adj, med, om)
    o.set_fp8(oc, osc)
    gi, gd, gn = g.search_arrays(Q, 10, 48, traversal=_lib.TRAVERSE_FP8)
    oi, od, on = o.search(Q, 10, 48, use_codes=True)
    assert np.array_equal(gn, on)
    same = np.mean([len(set(gi[i]) & set(oi[i])) / 10 for i in range(len(Q))])
    assert same >= 0.97, same
    qn = (Q.astype(np.float64) ** 2).sum(1)
    for i in range(len(Q)):
        for j in range(10):
            if gi[i, j] == oi[i, j]:
                xn = float((X[gi[i, j]].astype(np.float64) ** 2).sum())
                tol = 1e-5 * (qn[i] + xn) if metric == "l2" else 2e-5
                assert abs(float(gd[i, j]) - float(od[i, j])) <= tol, (i, j, gd[i, j], od[i, j])
    # with the FP32 rerank of the working set: exact distances, recall near FP32's
    ri, rd, rn = g.search_arrays(Q, 10, 48, traversal=_lib.TRAVERSE_FP8, rerank_size=48)
    fi, fd, fn = g.search_arrays(Q, 10, 48, traversal=_lib.TRAVERSE_F32)
    m = ri == fi
    assert np.array_equal(rd[m], fd[m])
    assert np.mean(m) >= 0.9
    g.close()


def test_packed_filters_equal_per_call_programs(small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    g = dg.FilteredDiskANN(X, adj, med, _labels(len(X)))
    fl = [FILTERS[i % len(FILTERS)] if i % 4 else dg.Filter.none() for i in range(len(Q))]
    a = g.search_arrays(Q, 10, 40, filters=fl)
    b = g.search_arrays(Q, 10, 40, filters=dg.pack_filters(fl))
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    g.close()


def test_bf16_after_row_and_adjacency_updates(oracle):
    """After rows and adjacency rows are rewritten in place
    (dg_index_update_rows), the BF16 copy and its per-row norms follow: BF16
    searches (with and without rerank) equal the oracle on the updated index."""
    from pydiskann_b200 import synth

    X = synth.mixture(4000, 128, 16, seed=52)
    Q = synth.mixture(300, 128, 16, seed=52, stream=synth.STREAM_QUERY)
    adj, med = oracle.build_vamana(X, 32, 64, 1.2, seed=8)
    adj = adj.reshape(len(X), -1).copy()
    ix = dg.DiskANN.from_graph(X, adj, med)
    ix.enable_bf16()
    rng = np.random.default_rng(52)
    # rows near the queries move (new integer values), other rows get new neighbours
    rows = np.unique(np.asarray(oracle.OracleIndex(X, adj, med).search(Q[:40], 5, 64)[0]).ravel())
    rows = rows[rows != med][:60].astype(np.int64)
    Xn = X.copy()
    for r in rows:
        Xn[r] = np.clip(np.round(X[r] + rng.normal(0, 30, X.shape[1])), 0, 255)
        assert _lib.lib().dg_index_update_rows(ix._h, int(r), 1, _lib.ptr(Xn[r:r + 1]), None, None) == _lib.DG_OK
    for r in rng.choice(len(X), 80, replace=False):
        row = adj[r].copy()
        row[: len(row) // 2] = rng.choice(len(X), len(row) // 2, replace=False)
        adj[r] = row
        assert _lib.lib().dg_index_update_rows(ix._h, int(r), 1, None, _lib.ptr(adj[r:r + 1]), None) == _lib.DG_OK
    o = oracle.OracleIndex(Xn, adj, med)
    o.set_bf16()
    for L, rr in ((40, 0), (64, 64)):
        assert_same(ix.search_arrays(Q, 10, L, traversal=_lib.TRAVERSE_BF16, rerank_size=rr),
                    o.search(Q, 10, L, rerank=rr, use_codes=True))
    ix.close()

