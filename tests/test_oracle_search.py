"""Oracle self-consistency on small seeded data (CPU)."""
import numpy as np

from kat_helpers import check_result_invariants


def test_graph_shape(small_data, small_graph):
    X, _ = small_data
    adj, med = small_graph
    assert adj.shape == (X.shape[0], 32)
    for u in range(0, X.shape[0], 97):
        row = [v for v in adj[u] if v != 0xFFFFFFFF]
        assert u not in row
        assert len(set(row)) == len(row)
        assert all(v < X.shape[0] for v in row)


def test_recall_and_invariants(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    idx = oracle.OracleIndex(X, adj, med)
    ids, ds, cnt = idx.search(Q, 10, 64)
    gt, _ = oracle.exact_knn(X, Q, 10)
    rec = np.mean([len(set(ids[i]) & set(gt[i])) / 10 for i in range(len(Q))])
    assert rec > 0.9, rec
    check_result_invariants([[(int(ids[i, j]), float(ds[i, j])) for j in range(cnt[i])] for i in range(len(Q))],
                            10, X.shape[0])


def test_batch_equals_single(oracle, small_data, small_graph):
    X, Q = small_data
    adj, med = small_graph
    idx = oracle.OracleIndex(X, adj, med)
    ids, ds, _ = idx.search(Q[:20], 10, 48)
    for i in range(20):
        i1, d1, _ = idx.search(Q[i:i + 1], 10, 48)
        assert (i1[0] == ids[i]).all() and (d1[0] == ds[i]).all()


def test_pq_adc_matches_decode(oracle, small_data):
    """src/pq.rs:458-484: table ADC equals the distance to the decoded vector."""
    X, Q = small_data
    rng = np.random.default_rng(3)
    cb = X[rng.choice(len(X), 256, replace=False)].reshape(256, 16, 8).transpose(1, 0, 2).copy()
    codes = oracle.pq_encode(X[:50], cb)
    lut = oracle.pq_lut(Q[0], cb)
    for i in range(50):
        dec = np.concatenate([cb[m, codes[i, m]] for m in range(16)])
        assert abs(oracle.pq_adc(lut, codes[i]) - float(((Q[0] - dec) ** 2).sum())) <= 1e-5 * max(1.0, float(((Q[0] - dec) ** 2).sum()))


def test_int8_asymmetric_within_one_percent(oracle):
    """src/sq.rs:398-419: int8 distance within 1% of the decoded distance."""
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (100, 64)).astype(np.float32)
    s, o = oracle.int8_train(X)
    codes = oracle.int8_encode(X, s, o)
    q = oracle.int8_encode(X[:1], s, o)[0]
    for i in range(1, 20):
        dq = q.astype(np.float32) * s + o
        dc = codes[i].astype(np.float32) * s + o
        ref = float(((dq - dc) ** 2).sum())
        assert abs(oracle.int8_distance(q, codes[i], s) - ref) <= 0.01 * ref + 1e-6


def test_rabitq_estimator_bound(oracle):
    """src/rabitq.rs:316-326: distance equals the asymmetric estimate; the error
    envelope holds for most candidates."""
    rng = np.random.default_rng(9)
    X = rng.standard_normal((300, 100)).astype(np.float32)
    P = oracle.rabitq_padded(100)
    assert P == 128
    cen = X.mean(0).astype(np.float32)
    signs = np.where(rng.integers(0, 2, 3 * P) == 1, 1, -1).astype(np.float32) / np.float32(np.sqrt(P))
    codes = oracle.rabitq_encode(X, P, cen, signs)
    assert codes.shape[1] == P // 8 + 8
    planes, k5 = oracle.rabitq_query(X[0], P, cen, signs)
    ok = 0
    for i in range(1, 300):
        est, err = oracle.rabitq_distance(planes, k5, codes[i], P, with_bound=True)
        assert est == oracle.rabitq_distance(planes, k5, codes[i], P)
        true = float(((X[0] - X[i]) ** 2).sum())
        ok += abs(true - est) <= err
    assert ok >= 0.9 * 299
