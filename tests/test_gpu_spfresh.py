"""SPFresh posting scans on the GPU vs the oracle's restatement of
Inner::search / search_rabitq (src/spfresh.rs:671-770) on the same posting
lists, after inserts and deletes.  Integer-valued data: distances are exact,
so ids, counts and distances must match bit for bit (cosine within 1e-5)."""
import numpy as np
import pytest

import pydiskann_b200 as dg
from pydiskann_b200 import synth

pytestmark = pytest.mark.gpu


def oracle_view(oracle, s):
    cent, live, lens, ids, codes = s.host_arrays(len(s.live_b))
    dele = np.zeros(max(s.next_id, 1), dtype=np.uint8)
    for i in s.deleted:
        dele[i] = 1
    raw = np.ascontiguousarray(s.raw[: s.next_id])
    v = oracle.Spfresh()
    keep = [cent, live, lens, ids, codes, dele, raw]
    p = oracle._p
    v.d, v.metric, v.num_blocks, v.block_cap = s.dim, s.metric, len(live), s.cap
    v.block_live, v.centroids, v.block_len, v.entry_ids = p(live), p(cent), p(lens), p(ids)
    v.entry_codes, v.code_size, v.deleted, v.next_id, v.raw = p(codes), s.codec.size, p(dele), s.next_id, p(raw)
    q = {None: oracle.Q_NONE, "f16": oracle.Q_F16, "int8": oracle.Q_INT8, "pq": oracle.Q_PQ, "rabitq": oracle.Q_RABITQ}
    v.quant = q[s.codec.kind]
    if s.codec.kind == "pq":
        cb = np.ascontiguousarray(s.codec.p["codebooks"], dtype=np.float32)
        keep.append(cb)
        v.pq_M, v.pq_K, v.pq_codebooks = cb.shape[0], cb.shape[1], p(cb)
    if s.codec.kind == "int8":
        v.int8_scale, v.int8_offset = s.codec.p["scale"], s.codec.p["offset"]
    if s.codec.kind == "rabitq":
        sg = np.ascontiguousarray(s.codec.p["signs"], dtype=np.float32)
        keep.append(sg)
        v.rq_padded, v.rq_signs = s.codec.p["padded"], p(sg)
    v.probe_ratio, v.rerank_size = s.probe_ratio, s.rerank_size
    return v, keep


CASES = [
    (None, "l2", 0, float("inf")),
    (None, "euclidean", 0, 1.5),
    ("int8", "l2", 20, float("inf")),
    ("int8", "l2", 0, float("inf")),
    ("f16", "l2", 15, 2.0),
    ("pq", "l2", 30, float("inf")),
    ("rabitq", "l2", 0, float("inf")),
    ("rabitq", "euclidean", 0, float("inf")),
]


@pytest.mark.parametrize("quant,metric,rerank,ratio", CASES)
def test_spfresh_scan_matches_oracle(oracle, quant, metric, rerank, ratio):
    X = synth.mixture(4000, 32, 40, seed=12, clip=False)
    s = dg.SPFresh.build(X, metric=metric, quantizer=quant, rerank_size=rerank, pq_subspaces=8, max_posting_size=40,
                         min_posting_size=8, probe_ratio=ratio, seed=2)
    s.insert(synth.mixture(500, 32, 40, seed=13, clip=False))
    s.delete(list(range(0, 4500, 9)))
    Q = synth.mixture(120, 32, 40, seed=12, stream=synth.STREAM_QUERY, clip=False)
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 1), (10, 6), (7, 40)):
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc), (k, nprobe)
        assert np.array_equal(gi, oi), (k, nprobe, np.nonzero((gi != oi).any(1))[0][:5])
        assert np.array_equal(gd, od), (k, nprobe)
    s.close()


@pytest.mark.parametrize("quant,metric", [("pq", "cosine"), ("pq", "dot"), ("rabitq", "cosine"), ("rabitq", "dot")])
def test_spfresh_decoded_metrics(oracle, quant, metric):
    """Cosine / dot over PQ and RaBitQ postings decode the code
    (src/spfresh.rs:344-354).  PQ decodes in coordinate order as the oracle does
    (bit-identical); RaBitQ sums the decoded coordinates across lanes, so ids
    agree except near-ties and distances within 1e-5 relative + 2e-6."""
    X, Q = synth.cosine(3000, 60, 64, seed=21)
    s = dg.SPFresh.build(X[:2500], metric=metric, quantizer=quant, rerank_size=0, pq_subspaces=8,
                         max_posting_size=40, min_posting_size=8, seed=5)
    s.insert(X[2500:])
    s.delete(list(range(0, 3000, 13)))
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 6), (7, 40)):
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc), (k, nprobe)
        if quant == "pq":
            assert np.array_equal(gi, oi) and np.array_equal(gd, od), (k, nprobe)
        else:
            same = np.mean([len(set(gi[i][:gc[i]]) & set(oi[i][:oc[i]])) / max(1, oc[i]) for i in range(len(Q))])
            assert same >= 0.98, same
            m = gi == oi
            assert np.all(np.abs(gd[m] - od[m]) <= 1e-5 * np.abs(od[m]) + 2e-6)
    s.close()


def test_spfresh_cosine_within_tolerance(oracle):
    X = synth.mixture(3000, 32, 30, seed=14, clip=False)
    s = dg.SPFresh.build(X, metric="cosine", max_posting_size=40, seed=3)
    Q = synth.mixture(80, 32, 30, seed=14, stream=synth.STREAM_QUERY, clip=False)
    view, keep = oracle_view(oracle, s)
    gi, gd, gc = s.search_arrays(Q, 10, 8)
    oi, od, oc = oracle.spfresh_search(view, Q, 10, 8)
    assert np.array_equal(gc, oc)
    assert np.mean([len(set(gi[i]) & set(oi[i])) / 10 for i in range(len(Q))]) >= 0.98
    same = gi == oi
    assert np.allclose(gd[same], od[same], rtol=1e-5, atol=1e-6)
    s.close()


def test_exhaustive_probe_is_exact_knn(oracle):
    """python/tests/test_spfresh.py:84-90: probing every posting returns the
    brute-force neighbours of the live vectors."""
    X = synth.mixture(3000, 32, 20, seed=15, clip=False)
    s = dg.SPFresh.build(X, max_posting_size=60, seed=4)
    s.delete(list(range(5, 3000, 11)))
    Q = synth.mixture(50, 32, 20, seed=15, stream=synth.STREAM_QUERY, clip=False)
    gi, gd, gc = s.search_arrays(Q, 10, 1024)
    live = np.array([i for i in range(3000) if i not in s.deleted])
    ei, ed = oracle.exact_knn(X[live], Q, 10)
    assert np.array_equal(gi.astype(np.int64), live[ei.astype(np.int64)])
    assert np.array_equal(gd, ed.astype(np.float32))
    # batch equals single (python/tests/test_spfresh.py:246-249)
    batch = s.search_batch(Q[:10], 10, 16)
    assert all(s.search(Q[i], 10, 16) == batch[i] for i in range(10))
    s.close()


def test_spfresh_api_errors():
    X = synth.mixture(500, 16, 4, seed=16, clip=False)
    s = dg.SPFresh.build(X, max_posting_size=32)
    with pytest.raises(ValueError):
        s.search([1.0, 2.0], 5, 2)
    with pytest.raises(RuntimeError):
        s.insert(np.zeros((2, 8), dtype=np.float32))
    assert s.stats()["live"] == 500
    s.close()


def test_bulk_load_scans_match_oracle(oracle):
    """bulk_load builds postings from an exact nearest-centroid assignment; the
    scans over them equal the oracle's, and updates continue afterwards."""
    X = synth.mixture(6000, 32, 40, seed=31, clip=False)
    s = dg.SPFresh.bulk_load(X, max_posting_size=40, seed=3)
    st = s.stats()
    assert st["live"] == 6000 and st["max_posting"] <= 40
    assert sorted(np.concatenate([s.ids[b] for b in range(len(s.live_b)) if s.live_b[b]]).tolist()) == list(range(6000))
    s.insert(synth.mixture(300, 32, 40, seed=32, clip=False))
    s.delete(list(range(0, 6300, 17)))
    Q = synth.mixture(100, 32, 40, seed=31, stream=synth.STREAM_QUERY, clip=False)
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 8), (10, 64)):
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od)
    s.close()


@pytest.mark.parametrize("metric", ["l2", "euclidean", "cosine"])
def test_many_postings_routing_kernel_matches_oracle(oracle, metric):
    """With >= 512 postings the routing distances come from a separate tiled
    kernel (each pair summed in coordinate order, as the oracle); ids, counts
    and distances stay bit-identical (cosine within 1e-5)."""
    if metric == "cosine":
        X, Q = synth.cosine(30000, 200, 48, seed=33)
    else:
        X = synth.mixture(30000, 48, 64, seed=33, clip=False)
        Q = synth.mixture(200, 48, 64, seed=33, stream=synth.STREAM_QUERY, clip=False)
    s = dg.SPFresh.bulk_load(X, metric=metric, max_posting_size=32, seed=6)
    assert s.stats()["postings"] >= 512
    s.delete(list(range(0, 30000, 23)))
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 4), (10, 40), (5, 300)):
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc), (k, nprobe)
        if metric == "cosine":
            assert np.mean(gi == oi) >= 0.98
            m = gi == oi
            assert np.allclose(gd[m], od[m], rtol=1e-5, atol=1e-6)
        else:
            assert np.array_equal(gi, oi) and np.array_equal(gd, od), (k, nprobe)
    s.close()


@pytest.mark.parametrize("metric", ["l2", "euclidean"])
def test_posting_major_scan_matches_oracle(oracle, metric):
    """Batches of >= 256 queries over >= 512 raw postings under L2 run the
    posting-major scan (pairs grouped by posting, one shared-memory load of a
    posting for all its queries, per-query merge; probes above 64 chosen by a
    radix select).  Results equal the oracle's and the query-major scan's (a
    batch of fewer than 256 queries), with tombstones, a probe_ratio cut and k
    up to 64."""
    X = synth.mixture(30000, 48, 64, seed=35, clip=False)
    Q = synth.mixture(700, 48, 64, seed=35, stream=synth.STREAM_QUERY, clip=False)
    s = dg.SPFresh.bulk_load(X, metric=metric, max_posting_size=32, seed=7)
    assert s.stats()["postings"] >= 512
    s.delete(list(range(0, 30000, 19)))
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 4), (10, 64), (64, 40), (1, 300)):
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od), (k, nprobe)
        qi, qd, qc = s.search_arrays(Q[:200], k, nprobe)  # query-major
        assert np.array_equal(qi, gi[:200]) and np.array_equal(qd, gd[:200]) and np.array_equal(qc, gc[:200])
    s.probe_ratio = 1.5
    view, keep = oracle_view(oracle, s)
    for nprobe in (64, 200):  # probes chosen by the sorted selection / the radix select
        gi, gd, gc = s.search_arrays(Q, 10, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, 10, nprobe)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od), nprobe
    s.close()


def test_rabitq_postings_reencoded_on_the_gpu(oracle):
    """RaBitQ posting codes are residuals against their posting's centroid, so
    splits and relocations re-encode them (Inner::encode,
    src/spfresh.rs:328-339).  The re-encode runs on the GPU encoder: after
    inserts that split postings, every entry's code equals the oracle's
    encode_with against its posting's current centroid."""
    X = synth.mixture(3000, 32, 30, seed=14, clip=False)
    s = dg.SPFresh.build(X, quantizer="rabitq", max_posting_size=40, min_posting_size=8, seed=3)
    s.insert(synth.mixture(800, 32, 30, seed=15, clip=False))
    s.delete(list(range(0, 3800, 13)))
    s.gc()
    P, signs = s.codec.p["padded"], s.codec.p["signs"]
    checked = 0
    for b in range(len(s.live_b)):
        if not s.live_b[b] or not len(s.ids[b]):
            continue
        want = oracle.rabitq_encode(s.raw[s.ids[b].astype(np.int64)], P, s.cent[b], signs)
        assert np.array_equal(s.codes[b], want), b
        checked += 1
    assert checked > 50
    s.close()


@pytest.mark.parametrize("d,metric", [(96, "l2"), (96, "euclidean"), (128, "l2"), (20, "l2")])
def test_tensor_core_routing_matches_oracle(oracle, d, metric):
    """Posting-major batches with n_probe <= 64 route on the tensor cores (FP16
    hi/lo products of centred, scaled vectors), then compute exact
    coordinate-order distances for every centroid within the error bound of
    each query's cut.  The probes, and so ids, counts and distances, equal the
    oracle's exact routing for several widths and a probe_ratio cut."""
    X = synth.mixture(30000, d, 64, seed=41, clip=False)
    Q = synth.mixture(600, d, 64, seed=41, stream=synth.STREAM_QUERY, clip=False)
    s = dg.SPFresh.bulk_load(X, metric=metric, max_posting_size=32, seed=8)
    assert s.stats()["postings"] >= 512
    s.delete(list(range(0, 30000, 29)))
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 16), (10, 64), (32, 33), (1, 1)):
        if 600 * nprobe < 16 * s.stats()["postings"]:
            continue  # below the posting-major threshold
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od), (k, nprobe)
    s.probe_ratio = 1.3
    view, keep = oracle_view(oracle, s)
    gi, gd, gc = s.search_arrays(Q, 10, 64)
    oi, od, oc = oracle.spfresh_search(view, Q, 10, 64)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od)
    s.close()


def test_tensor_core_routing_wide_bound_falls_back_exactly(oracle):
    """Two clusters 2e5 apart along one axis: after centring, every norm is
    about 1e10, so the tensor-core error bound covers every centroid of a
    query's half and the candidates outgrow a query's list.  Those queries
    fall back to exact distances for every live centroid; results still equal
    the oracle's."""
    rng = np.random.default_rng(5)
    X = synth.mixture(30000, 32, 64, seed=43, clip=False)
    X[:, 0] += np.where(rng.random(30000) < 0.5, -1e5, 1e5).astype(np.float32)
    Q = synth.mixture(600, 32, 64, seed=43, stream=synth.STREAM_QUERY, clip=False)
    Q[:, 0] += np.where(rng.random(600) < 0.5, -1e5, 1e5).astype(np.float32)
    s = dg.SPFresh.bulk_load(X, metric="l2", max_posting_size=32, seed=9)
    assert s.stats()["postings"] >= 512
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 64), (10, 40)):
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od), (k, nprobe)
    s.close()


@pytest.mark.parametrize("quant,metric", [("int8", "l2"), ("pq", "l2"), ("rabitq", "l2"), ("rabitq", "euclidean"),
                                          (None, "euclidean")])
def test_tensor_core_routing_feeds_query_major_scan(oracle, quant, metric):
    """Batches of >= 256 queries that probe too few postings for the
    posting-major scan still route on the tensor cores; the query-major scan
    then takes the probes as given.  Quantized postings (codes scanned, exact
    re-check or rerank as configured) give the oracle's results bit for bit."""
    X = synth.mixture(30000, 48, 64, seed=45, clip=False)
    Q = synth.mixture(300, 48, 64, seed=45, stream=synth.STREAM_QUERY, clip=False)
    kw = {} if quant is None else {"quantizer": quant}
    s = dg.SPFresh.bulk_load(X, metric=metric, max_posting_size=32, seed=10, **kw)
    assert s.stats()["postings"] >= 512
    s.delete(list(range(0, 30000, 31)))
    view, keep = oracle_view(oracle, s)
    for k, nprobe in ((10, 4), (10, 20)):
        assert 300 * nprobe < 16 * s.stats()["postings"]  # query-major
        gi, gd, gc = s.search_arrays(Q, k, nprobe)
        oi, od, oc = oracle.spfresh_search(view, Q, k, nprobe)
        assert np.array_equal(gc, oc) and np.array_equal(gi, oi) and np.array_equal(gd, od), (k, nprobe)
    s.close()
