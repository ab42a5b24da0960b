"""Pins the CPU oracle to the reference test-suite's known answers."""
import numpy as np
import pytest

from kat_helpers import build_filter, check_index_kats, check_result_invariants, load_kats


@pytest.fixture(scope="module")
def kats():
    return load_kats()


def test_beam_search_small_graph(oracle, kats):
    c = kats["beam_search_small_graph"]
    pos = np.asarray(c["positions"], dtype=np.float32)
    q = np.asarray(c["query"], dtype=np.float32)
    nd = np.sqrt(((pos - q) ** 2).sum(1)).astype(np.float32)
    adj = np.asarray(c["neighbors"], dtype=np.uint32)
    r = oracle.beam_search_table(adj, nd, c["start"], c["beam_width"], c["k"])
    assert len(r) == c["expect_len"]
    assert [i for i, _ in r[:2]] == c["expect_prefix"]
    assert [d for _, d in r] == sorted(d for _, d in r)


def test_beam_search_with_filter(oracle, kats):
    c = kats["beam_search_with_filter"]
    pos = np.asarray(c["positions"], dtype=np.float32)
    q = np.asarray(c["query"], dtype=np.float32)
    nd = np.sqrt(((pos - q) ** 2).sum(1)).astype(np.float32)
    adj = np.asarray(c["neighbors"], dtype=np.uint32)
    allow = np.array([1 if i in c["allowed"] else 0 for i in range(len(pos))], dtype=np.uint8)
    r = oracle.beam_search_table(adj, nd, c["start"], c["beam_width"], c["k"], allow=allow, filtered=True,
                                 expanded=c["expanded_beam"], max_iter=c["max_iterations"],
                                 early=c["early_term_factor"])
    ids = {i for i, _ in r}
    assert all(i % 2 == 1 for i in ids)
    assert set(c["expect_contains"]) <= ids


def test_prune_alpha(oracle, kats):
    c = kats["prune_alpha"]
    X = np.asarray(c["vectors"], dtype=np.float32)
    ids = c["cands"]
    d = [oracle.distance(oracle.L2, X[c["node"]], X[i]) for i in ids]
    pr = oracle.robust_prune(c["node"], ids, d, X, c["max_degree"], c["alpha"], oracle.L2)
    assert set(c["expect_contains"]) <= set(pr)


def test_prune_max_degree(oracle, kats):
    c = kats["prune_max_degree"]
    X = np.asarray(c["vectors"], dtype=np.float32)
    ids = c["cands"]
    d = [oracle.distance(oracle.L2, X[c["node"]], X[i]) for i in ids]
    for R, want in c["degree_to_len"]:
        assert len(oracle.robust_prune(c["node"], ids, d, X, R, c["alpha"], oracle.L2)) == want


def _oracle_build_and_search(oracle):
    def run(vectors, metric, R, Lb, alpha, queries, k, L):
        m = oracle.METRICS[metric]
        X = np.asarray(vectors, dtype=np.float32)
        adj, med = oracle.build_vamana(X, R, Lb, alpha, seed=1, metric=m)
        idx = oracle.OracleIndex(X, adj, med, m)
        ids, ds, cnt = idx.search(np.asarray(queries, dtype=np.float32), k, L)
        return [[(int(ids[i, j]), float(ds[i, j])) for j in range(cnt[i])] for i in range(len(cnt))]

    return run


def test_index_kats(oracle, kats):
    check_index_kats(kats, _oracle_build_and_search(oracle))


def test_filter_truth_tables(oracle, kats):
    from pydiskann_b200 import Filter

    for case in kats["filters"]:
        f = build_filter(case["filter"], Filter)
        ops, pool = f.program()
        for lab in case["true"]:
            assert f.matches(lab)
            assert oracle.filter_matches(ops, pool, lab if lab else [0])
        for lab in case["false"]:
            assert not f.matches(lab)
            if lab:
                assert not oracle.filter_matches(ops, pool, lab)


def test_rabitq_sizes(oracle, kats):
    from pydiskann_b200 import rabitq_padded

    for d, p in kats["rabitq_sizes"]["padded"]:
        assert oracle.rabitq_padded(d) == p
        assert rabitq_padded(d) == p
    for p, cs in kats["rabitq_sizes"]["code_size"]:
        assert p // 8 + 8 == cs


def test_k_greater_than_n(oracle):
    rng = np.random.default_rng(200)
    X = rng.random((5, 16), dtype=np.float32)
    adj, med = oracle.build_vamana(X, 64, 128, 1.2, seed=2)
    idx = oracle.OracleIndex(X, adj, med)
    ids, ds, cnt = idx.search(X[:1], 100, 64)
    rows = [[(int(ids[0, j]), float(ds[0, j])) for j in range(cnt[0])]]
    check_result_invariants(rows, 100, 5)
