"""Indexes opened from the reference's file formats search like the indexes
they were written from (pydiskann_b200/formats.py on the GPU path).

A core file assembled byte by byte from the reference's layout (src/lib.rs:
355-680) opens with DiskANN.open and searches bit-identically to the oracle
over the same arrays; build(path=...) / save_quantized / to_bytes write files
that open back into indexes whose codes and results are identical.
Tolerance: none (ids, counts, distances and code bytes bit-identical).
"""
import struct

import numpy as np
import pytest

import pydiskann_b200 as dg
from pydiskann_b200 import formats as F

pytestmark = pytest.mark.gpu


def _same(a, b, Q, k=10, L=64, **kw):
    ia, da, ca = a.search_arrays(Q, k, L, **kw)
    ib, db, cb = b.search_arrays(Q, k, L, **kw)
    assert np.array_equal(ca, cb) and np.array_equal(ia, ib) and np.array_equal(da, db)


def test_hand_built_core_file_matches_oracle(tmp_path, small_data, small_graph, oracle):
    X, Q = small_data
    adj, med = small_graph
    n, d = X.shape
    R = adj.shape[1]
    name = b"diskann_rs::metric::DistL2Sq"
    md = struct.pack("<QQQIQQ", d, n, R, med, 1 << 20, (1 << 20) + n * d * 4) + struct.pack("<Q", len(name)) + name
    head = struct.pack("<IIQ", 0x44414E4E, 1, len(md)) + md
    p = tmp_path / "ref.idx"
    p.write_bytes(head + bytes((1 << 20) - len(head)) + X.astype("<f4").tobytes() + adj.astype("<u4").tobytes())
    idx = dg.DiskANN.open(str(p))
    assert (idx.num_vectors, idx.dim, idx.max_degree, idx.medoid_id) == (n, d, R, med)
    ids, ds, cnt = idx.search_arrays(Q[:64], 10, 64)
    oi, od, oc = oracle.OracleIndex(X, adj, med).search(Q[:64], 10, 64)
    assert np.array_equal(cnt, oc) and np.array_equal(ids, oi) and np.array_equal(ds, od)
    assert idx.to_bytes() == p.read_bytes()
    idx.close()


def test_diskann_build_open_from_bytes(tmp_path, small_data):
    X, Q = small_data
    p = str(tmp_path / "a.idx")
    built = dg.DiskANN.build(X[:1500], p, max_degree=24, build_beam_width=48)
    opened = dg.DiskANN.open(p)
    _same(built, opened, Q)
    again = dg.DiskANN.from_bytes(opened.to_bytes())
    _same(built, again, Q)
    assert opened.get_vector(7) == built.get_vector(7)
    with pytest.warns(RuntimeWarning, match="recorded distance"):
        dg.DiskANN.open(p, metric="dot").close()
    with pytest.raises(ValueError):
        dg.DiskANN.open(p, metric="hamming")
    for i in (built, opened, again):
        i.close()


@pytest.mark.parametrize("quantizer", ["pq", "int8", "f16", "rabitq"])
def test_quantized_sidecar_roundtrip(tmp_path, small_data, quantizer):
    X, Q = small_data
    base, side = str(tmp_path / "q.idx"), str(tmp_path / "q.qann")
    q = dg.QuantizedDiskANN.build(X[:1500], base, quantizer=quantizer, rerank_size=30, pq_subspaces=16,
                                  max_degree=24, build_beam_width=48)
    q.save_quantized(side)
    st, codes = F.read_sidecar(side, 1500)
    assert st.kind == quantizer and np.array_equal(codes, q.codes())
    o = dg.QuantizedDiskANN.open(base, side, rerank_size=30)
    assert np.array_equal(o.codes(), q.codes())
    _same(q, o, Q)
    _same(q, o, Q, rerank_size=0)
    b = dg.QuantizedDiskANN.from_bytes(q.to_bytes(), rerank_size=30)
    _same(q, b, Q)
    if quantizer == "f16":  # codes from the sidecar are the RNE f16 bit patterns
        assert np.array_equal(codes.view("<u2"), X[:1500].astype(np.float16).view(np.uint16))
    for i in (q, o, b):
        i.close()


def test_quantized_open_errors(tmp_path, small_data):
    X, _ = small_data
    base, side = str(tmp_path / "e.idx"), str(tmp_path / "e.qann")
    q = dg.QuantizedDiskANN.build(X[:800], base, quantizer="int8", max_degree=16, build_beam_width=32)
    q.save_quantized(side)
    q.close()
    F.write_core(str(tmp_path / "small.idx"), X[:700], np.zeros((700, 4), np.uint32), 0)
    with pytest.raises(RuntimeError, match="Sidecar has 800 vectors, base index has 700"):
        dg.QuantizedDiskANN.open(str(tmp_path / "small.idx"), side)


def test_filtered_build_open_from_bytes(tmp_path, small_data):
    X, Q = small_data
    n = 1500
    rng = np.random.default_rng(4)
    labels = np.stack([np.arange(n) % 4, rng.integers(0, 50, n)], 1).astype(np.uint64)
    p = str(tmp_path / "f")
    built = dg.FilteredDiskANN.build(X[:n], labels, p, max_degree=24, build_beam_width=48)
    opened = dg.FilteredDiskANN.open(p)
    assert np.array_equal(F.read_labels(p + ".labels"), labels)
    flt = dg.Filter.and_([dg.Filter.eq(0, 1), dg.Filter.range(1, 5, 40)])
    _same(built, opened, Q, filters=flt)
    again = dg.FilteredDiskANN.from_bytes(opened.to_bytes())
    _same(built, again, Q, filters=flt)
    assert again.count_matching(flt) == built.count_matching(flt)
    F.write_labels(p + ".labels", labels[:10])
    with pytest.raises(RuntimeError, match=r"Labels count \(10\) != index vectors \(1500\)"):
        dg.FilteredDiskANN.open(p)
    for i in (built, opened, again):
        i.close()


@pytest.mark.parametrize("quantizer", [None, "int8", "pq", "rabitq"])
def test_spfresh_save_open(tmp_path, small_data, quantizer):
    """SPFresh::save / open (src/spfresh.rs:819-859): the reopened index scans
    the same postings and returns the same results, and keeps updating."""
    X, Q = small_data
    p = str(tmp_path / "sp")
    s = dg.SPFresh.build(X[:3000], p, quantizer=quantizer, rerank_size=20 if quantizer else 0,
                         pq_subspaces=16, max_posting_size=64)
    s.delete(list(range(0, 3000, 7)))
    s.save()
    t = dg.SPFresh.open(p)
    for nprobe in (4, 16):
        a = s.search_arrays(Q, 10, nprobe)
        b = t.search_arrays(Q, 10, nprobe)
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x), np.asarray(y))
    ids = t.insert(X[3000:3200])
    assert ids == list(range(3000, 3200))
    assert 3100 in [i for i, _ in t.search_with_dists(X[3100], 5, 16)]
    s.close()
    t.close()
