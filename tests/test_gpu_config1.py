"""Parity on the plain Vamana configuration at its full size: 100k x 128
integer-valued vectors from a 64-centre Gaussian mixture (sigma 20, clipped to
[0, 255], seed 0), 1k queries drawn the same way, graph R=32, L_build=64,
alpha=1.2, search L=64, k=10.

The graph built on the GPU equals the oracle's build of the same seed, and the
batched GPU search over it -- plain FP32, BF16 rows + FP32 rerank of the top L,
int8 codes + FP32 rerank -- returns the oracle's ids, distances and counts bit
for bit (every partial sum of these integer-valued rows is exact in FP32).
Recall@10 is checked against exact FP64 kNN.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, NQ, R, L_BUILD, ALPHA, L, K = 100_000, 1_000, 32, 64, 1.2, 64, 10


@pytest.fixture(scope="module")
def cfg1(oracle):
    import pydiskann_b200 as dg
    from pydiskann_b200 import synth

    X, Q = synth.plain(N, NQ, 128, 0)
    med = dg.medoid(X)
    assert med == oracle.medoid(X)
    adj, _ = dg.build_graph(X, R, L_BUILD, ALPHA, seed=0, medoid_id=med)
    gt, _ = oracle.exact_knn(X, Q, K)
    return X, Q, adj, med, gt


def test_graph_build_equals_oracle_build(oracle, cfg1):
    X, _, adj, med, _ = cfg1
    oadj, _ = oracle.build_vamana(X, R, L_BUILD, ALPHA, seed=0, medoid_id=med)
    diff = np.nonzero((adj != oadj).any(1))[0]
    assert diff.size == 0, f"{diff.size} adjacency rows differ, first {diff[:5]}"


@pytest.mark.parametrize("variant", ["fp32", "bf16_rerank", "int8_rerank"])
def test_search_bit_exact_vs_oracle(oracle, cfg1, variant):
    import pydiskann_b200 as dg
    from pydiskann_b200 import _lib

    X, Q, adj, med, gt = cfg1
    o = oracle.OracleIndex(X, adj, med)
    if variant == "fp32":
        ix = dg.DiskANN.from_graph(X, adj, med)
        got = ix.search_arrays(Q, K, L, with_stats=True)
        want = o.search(Q, K, L, with_stats=True)
    elif variant == "bf16_rerank":
        ix = dg.DiskANN.from_graph(X, adj, med)
        ix.enable_bf16()
        got = ix.search_arrays(Q, K, L, traversal=_lib.TRAVERSE_BF16, rerank_size=L, with_stats=True)
        o.set_bf16()
        want = o.search(Q, K, L, rerank=L, use_codes=True, with_stats=True)
    else:
        ix = dg.QuantizedDiskANN(X, adj, med)
        sc, off = dg.int8_params(X)
        ix.attach_int8(sc, off)
        got = ix.search_arrays(Q, K, L, rerank_size=L, with_stats=True)
        o.set_int8(sc, off, oracle.int8_encode(X, sc, off))
        want = o.search(Q, K, L, rerank=L, use_codes=True, with_stats=True)
    ix.close()
    gi, gd, gc, gs = got
    oi, od, oc, os_ = want
    assert np.array_equal(gc, oc)
    assert np.array_equal(gi, oi), f"{int((gi != oi).any(1).sum())} queries differ"
    assert np.array_equal(gd, od)
    assert np.array_equal(gs[:, 0], os_[:, 0])  # expansions: the same search
    assert (gs[:, 1] >= os_[:, 1]).all()  # forgotten visited ids are evaluated again
    hits = sum(len(set(gi[i, :K].tolist()) & set(gt[i, :K].tolist())) for i in range(NQ))
    assert hits / (NQ * K) >= 0.95
