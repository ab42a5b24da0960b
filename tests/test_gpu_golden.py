"""The GPU path against the reference test-suite's known answers, and the GPU
graph build / medoid / exact kNN against the oracle's."""
import numpy as np
import pytest

import pydiskann_b200 as dg
from kat_helpers import build_filter, check_index_kats, check_result_invariants, load_kats

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kats():
    return load_kats()


def test_beam_search_small_graph(kats):
    c = kats["beam_search_small_graph"]
    idx = dg.DiskANN.from_graph(c["positions"], c["neighbors"], c["start"][0], metric=c["metric"])
    r = idx.search_with_dists(c["query"], c["k"], c["beam_width"])
    assert len(r) == c["expect_len"]
    assert [i for i, _ in r[:2]] == c["expect_prefix"]


def test_beam_search_with_filter(kats):
    c = kats["beam_search_with_filter"]
    labels = [[i % 2] for i in range(len(c["positions"]))]
    idx = dg.FilteredDiskANN(c["positions"], c["neighbors"], c["start"][0], labels, metric=c["metric"])
    r = idx.search_filtered_with_dists(c["query"], dg.Filter.eq(0, 1), c["k"], c["beam_width"])
    ids = {i for i, _ in r}
    assert all(i % 2 == 1 for i in ids)
    assert set(c["expect_contains"]) <= ids


def test_index_kats(kats):
    def run(vectors, metric, R, Lb, alpha, queries, k, L):
        idx = dg.DiskANN.build(vectors, metric=metric, max_degree=R, build_beam_width=Lb, alpha=alpha, seed=1)
        return [idx.search_with_dists(q, k, L) for q in queries]

    check_index_kats(kats, run)


def test_filter_truth_tables_on_device(kats):
    """Each truth-table row becomes a one-vector index whose filtered search
    must return the vector exactly when the filter matches."""
    for case in kats["filters"]:
        f = build_filter(case["filter"], dg.Filter)
        for lab, want in [(l, True) for l in case["true"]] + [(l, False) for l in case["false"]]:
            if not lab:
                continue
            idx = dg.FilteredDiskANN([[0.0, 0.0]], [[0xFFFFFFFF]], 0, [lab])
            got = idx.search_filtered([0.0, 0.0], f, 1, 4)
            assert (got == [0]) == want, (case["filter"], lab)
            assert idx.count_matching(f) == int(want)
            idx.close()


@pytest.mark.parametrize("n,d,R,Lb", [(1500, 32, 16, 32), (3000, 128, 32, 64)])
def test_build_matches_oracle(oracle, n, d, R, Lb):
    from pydiskann_b200 import synth

    X = synth.mixture(n, d, 16, seed=21)
    med = oracle.medoid(X)
    assert dg.medoid(X) == med
    oadj, _ = oracle.build_vamana(X, R, Lb, 1.2, seed=5, medoid_id=med)
    gadj, gmed = dg.build_graph(X, R, Lb, 1.2, seed=5, medoid_id=med)
    assert gmed == med
    diff = np.nonzero((gadj != oadj).any(1))[0]
    assert len(diff) == 0, (len(diff), diff[:5], gadj[diff[0]], oadj[diff[0]])


def test_exact_knn_matches_oracle(oracle, small_data):
    X, Q = small_data
    gi, gd = dg.exact_knn(X, Q[:64], 20)
    oi, od = oracle.exact_knn(X, Q[:64], 20)
    assert np.array_equal(gi, oi)
    assert np.array_equal(gd, od.astype(np.float32))


def test_recall_and_invariants_gpu_built(small_data):
    X, Q = small_data
    idx = dg.DiskANN.build(X, max_degree=32, build_beam_width=64, seed=3)
    ids, ds, cnt = idx.search_arrays(Q, 10, 64)
    gt, _ = dg.exact_knn(X, Q, 10)
    rec = np.mean([len(set(ids[i]) & set(gt[i])) / 10 for i in range(len(Q))])
    assert rec > 0.9
    check_result_invariants([[(int(ids[i, j]), float(ds[i, j])) for j in range(cnt[i])] for i in range(len(Q))],
                            10, len(X))
    # batch equals single (tests/correctness.rs:1042-1069)
    batch = idx.search_batch(Q[:16], 10, 64)
    for i in range(16):
        assert idx.search(Q[i], 10, 64) == batch[i]
