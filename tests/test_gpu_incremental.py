"""Base + delta (IncrementalDiskANN) search on the GPU against the oracle.

The oracle's restatement of IncrementalDiskANN::search_with_dists /
search_filtered_with_dists (src/incremental.rs:934-1070) runs over the same
unified view (base rows, delta rows, delta adjacency shifted by base_count)
with the same seeds, tombstones and labels.  Tolerance: none (ids, counts and
FP32 distances bit-identical; integer-valued data).
"""
import numpy as np
import pytest

import pydiskann_b200 as dg
from pydiskann_b200.incremental import DELTA_ID_OFFSET

pytestmark = pytest.mark.gpu
PAD = 0xFFFFFFFF


def _unified(ix):
    """Host copy of the unified view: vectors, adjacency, seeds, dead flags."""
    nb, dn = ix.base_count, ix._dn
    X = np.concatenate([ix._bX, ix._dX[:dn]])
    R = max(ix._bA.shape[1], ix._dR)
    A = np.full((nb + dn, R), PAD, np.uint32)
    A[:nb, : ix._bA.shape[1]] = ix._bA
    dA = ix._dA[:dn]
    A[nb:, : dA.shape[1]] = np.where(dA != PAD, dA + nb, PAD)
    seeds = [ix._bmed] + ([nb + ix._ep] if ix._ep >= 0 else [])
    dead = np.zeros(nb + dn, np.uint8)
    for g in ix.tombstones:
        r = ix._row_of(g)
        if r is not None:
            dead[r] = 1
    return X, A, seeds, dead


def _check(ix, oracle, Q, k, L, flt=None, labels=None):
    X, A, seeds, dead = _unified(ix)
    o = oracle.OracleIndex(X, A, seeds[0])
    ops, pool = (None, ())
    if flt is not None:
        o.set_labels(labels)
        ops, pool = flt.program()
    oi, od, oc = o.incremental_search(Q, k, L, seeds, dead, len(ix.tombstones), ops, pool)
    gi, gd, gc = ix.search_arrays(Q, k, L, filters=flt)
    nb = ix.base_count
    want = oi.astype(np.uint64)
    dl = (oi != PAD) & (oi >= nb)
    want[dl] = np.uint64(DELTA_ID_OFFSET) + (oi[dl].astype(np.uint64) - np.uint64(nb))
    assert np.array_equal(gc, oc)
    for q in range(len(Q)):
        c = int(oc[q])
        assert np.array_equal(gi[q, :c], want[q, :c]), q
        assert np.array_equal(gd[q, :c], od[q, :c]), q


@pytest.fixture()
def inc(small_data, small_graph):
    X, _ = small_data
    adj, med = small_graph
    # the base is the first 3000 rows with a graph over them
    import oracle as o

    base = X[:3000]
    badj, bmed = o.build_vamana(base, R=32, L_build=64, alpha=1.2, seed=3)
    ix = dg.IncrementalDiskANN(base, badj, bmed)
    yield ix, X
    ix.close()


def test_two_seeds_no_tombstones(inc, small_data, oracle):
    ix, X = inc
    _, Q = small_data
    ids = ix.add_vectors(X[3000:3300])
    assert ids[0] == DELTA_ID_OFFSET and ids[-1] == DELTA_ID_OFFSET + 299
    ix.add_vectors(X[3300:3700])
    for L in (1, 2, 16, 64, 200):
        _check(ix, oracle, Q, 10, L)
    # results merge both layers.  (Base and delta graphs share no edges in the
    # reference's unified view, so a query does not always reach its delta
    # neighbours when base candidates fill the beam first; the oracle agrees.)
    ids, _, cnt = ix.search_arrays(X[3000:3700:7], 10, 128)
    found = [int(i) for q in range(len(cnt)) for i in ids[q, : cnt[q]]]
    assert any(i >= DELTA_ID_OFFSET for i in found) and any(i < DELTA_ID_OFFSET for i in found)


def test_tombstones_config_and_exclusion(inc, small_data, oracle):
    ix, X = inc
    _, Q = small_data
    ix.add_vectors(X[3000:3500])
    gone = list(range(0, 3000, 11)) + [DELTA_ID_OFFSET + j for j in range(0, 500, 7)]
    gone.append(DELTA_ID_OFFSET + 900)  # not inserted yet: counted, and dead once it exists
    ix.delete_vectors(gone)
    for L in (8, 40, 128):
        for k in (1, 10):
            _check(ix, oracle, Q, k, L)
    ids, _, cnt = ix.search_arrays(Q, 10, 64)
    got = {int(i) for q in range(len(Q)) for i in ids[q, : cnt[q]]}
    assert not got & set(gone)
    ix.add_vectors(X[3500:3901])  # creates local id 900 (already tombstoned)
    _check(ix, oracle, Q, 10, 64)
    assert DELTA_ID_OFFSET + 900 not in ix.search(X[3900], 10, 64)
    st = ix.stats()
    assert st["delta_vectors"] == 901 and st["tombstones"] == len(set(gone))


def test_labels_filter(small_data, oracle):
    import oracle as o

    X, Q = small_data
    base = X[:2500]
    badj, bmed = o.build_vamana(base, R=24, L_build=48, alpha=1.2, seed=4)
    rng = np.random.default_rng(9)
    lab = np.stack([np.arange(4000) % 3, rng.integers(0, 20, 4000)], 1).astype(np.uint64)
    ix = dg.IncrementalDiskANN(base, badj, bmed, labels=lab[:2500])
    ix.add_vectors_with_labels(X[2500:3200], lab[2500:3200])
    ix.add_vectors(X[3200:3400])  # labels default to zeros
    ix.delete_vectors(range(0, 2500, 13))
    flt = dg.Filter.and_([dg.Filter.eq(0, 1), dg.Filter.lt(1, 12)])
    full = np.concatenate([lab[:3200], np.zeros((200, 2), np.uint64)])
    for L in (16, 64):
        _check(ix, oracle, Q, 10, L, flt, full)
    ix.close()


def test_growth_compaction_and_bytes(inc, small_data, oracle):
    ix, X = inc
    _, Q = small_data
    for c in range(3000, 4000, 250):  # grows past the initial 1024 spare rows
        ix.add_vectors(X[c:c + 250])
    ix.add_vectors(X[:200] + 1.0)
    ix.delete_vectors([5, 6, DELTA_ID_OFFSET + 3])
    _check(ix, oracle, Q, 10, 64)
    blob = ix.to_bytes()
    back = dg.IncrementalDiskANN.from_bytes(blob)
    a = ix.search_arrays(Q, 10, 64)
    b = back.search_arrays(Q, 10, 64)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert back.to_bytes() == blob
    back.close()
    live = ix.stats()["total_live"]
    ix.compact()
    st = ix.stats()
    assert st["base_vectors"] == live and st["delta_vectors"] == 0 and st["tombstones"] == 0
    got = ix.search(X[3100], 1, 64)
    assert len(got) == 1 and got[0] < DELTA_ID_OFFSET


@pytest.mark.parametrize("quantizer", ["int8", "pq", "rabitq", "f16"])
def test_quantized_base(small_data, oracle, quantizer):
    """build_quantized_* (src/incremental.rs:674-827): base rows are scored by
    their codes, delta rows exactly, then the FP32 rerank; the oracle runs the
    same search over the same codes with tombstones in play."""
    import oracle as o

    X, Q = small_data
    base = X[:2500]
    badj, bmed = o.build_vamana(base, R=24, L_build=48, alpha=1.2, seed=5)
    qp = {}
    if quantizer == "int8":
        qp["scale"], qp["offset"] = dg.int8_params(base)
    elif quantizer == "pq":
        qp["codebooks"] = dg.pq_train(base, 16, 256, 8, 2500, seed=2)
    elif quantizer == "rabitq":
        qp["centroid"], qp["signs"] = dg.rabitq_params(base, seed=2)
    ix = dg.IncrementalDiskANN(base, badj, bmed, quantizer=quantizer, qparams=qp, rerank_size=24)
    ix.add_vectors(X[2500:3100])
    ix.delete_vectors(list(range(0, 2500, 17)) + [DELTA_ID_OFFSET + 5])
    X_u, A, seeds, dead = _unified(ix)
    ov = oracle.OracleIndex(X_u, A, seeds[0])
    codes = np.zeros((len(X_u), ix._ix.codes().shape[1]), np.uint8)
    codes[: ix.base_count] = ix._ix.codes()[: ix.base_count]
    if quantizer == "int8":
        ov.set_int8(qp["scale"], qp["offset"], codes)
    elif quantizer == "pq":
        ov.set_pq(qp["codebooks"], codes)
    elif quantizer == "rabitq":
        ov.set_rabitq(dg.rabitq_padded(X.shape[1]), qp["centroid"], qp["signs"], codes)
    else:
        ov.set_f16(codes.view(np.uint16))
    for rr in (0, 24):
        oi, od, oc = ov.incremental_search(Q, 10, 48, seeds, dead, len(ix.tombstones), use_codes=True, rerank=rr,
                                           code_limit=ix.base_count)
        gi, gd, gc = ix.search_arrays(Q, 10, 48, rerank_size=rr)
        nb = ix.base_count
        want = oi.astype(np.uint64)
        dl = (oi != PAD) & (oi >= nb)
        want[dl] = np.uint64(DELTA_ID_OFFSET) + (oi[dl].astype(np.uint64) - np.uint64(nb))
        assert np.array_equal(gc, oc)
        assert np.array_equal(gi, np.where(oi == PAD, np.uint64(PAD), want)), quantizer
        assert np.array_equal(gd, od), quantizer
    back = dg.IncrementalDiskANN.from_bytes(ix.to_bytes())
    for x, y in zip(ix.search_arrays(Q, 10, 48), back.search_arrays(Q, 10, 48)):
        assert np.array_equal(x, y)
    back.close()
    ix.close()

