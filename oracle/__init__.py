"""CPU oracle for the pydiskann_b200 search kernels -- TEST INFRASTRUCTURE ONLY.

ctypes view of ``oracle/_build/libdgoracle.so`` (built from ``dgoracle.cpp`` by
``oracle/Makefile``).  The oracle restates the diskann-rs 0.5.0 search path on
the CPU (file:line citations live in dgoracle.cpp).  Only the tests, the smoke
check and the CPU-baseline leg of bench.py import this module; the product
package never does.

Parity status: pinned against the reference test-suite's known-answer tests
(tests/golden/); the reference binary is not buildable here (Rust crate, no
Rust toolchain), so no numeric golden outputs of the reference itself exist.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libdgoracle.so")

L2SQ, L2, COSINE, DOT = 0, 1, 2, 3
Q_NONE, Q_PQ, Q_INT8, Q_RABITQ, Q_F16, Q_FP8, Q_BF16 = 0, 1, 2, 3, 4, 5, 6
PAD = 0xFFFFFFFF
METRICS = {"l2": L2SQ, "l2sq": L2SQ, "euclidean": L2, "cosine": COSINE, "dot": DOT}


def build() -> str:
    """Compile the oracle library (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


_lib = None
_native = None
_SO_NATIVE = os.path.join(_HERE, "_build", "libdgoracle_native.so")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
            os.path.join(_HERE, "dgoracle.cpp")
        ):
            build()
        _lib = C.CDLL(_SO)
        _declare(_lib)
    return _lib


def lib_native():
    """The same oracle compiled for the machine running it (-O3 -march=native),
    built there on first use: the CPU timing legs of the bench use it."""
    global _native
    if _native is None:
        subprocess.run(["make", "-s", "-C", _HERE, "native"], check=True)
        _native = C.CDLL(_SO_NATIVE)
        _declare(_native)
    return _native


class FilterOp(C.Structure):
    _fields_ = [("op", C.c_uint32), ("field", C.c_uint32), ("a", C.c_uint64), ("b", C.c_uint64)]


class Index(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("d", C.c_uint32), ("R", C.c_uint32), ("medoid", C.c_uint32),
        ("metric", C.c_int32), ("vectors", C.c_void_p), ("adjacency", C.c_void_p),
        ("quant", C.c_int32), ("codes", C.c_void_p), ("code_size", C.c_uint32),
        ("pq_M", C.c_uint32), ("pq_K", C.c_uint32), ("pq_codebooks", C.c_void_p),
        ("int8_scale", C.c_float), ("int8_offset", C.c_float), ("rq_padded", C.c_uint32),
        ("rq_centroid", C.c_void_p), ("rq_signs", C.c_void_p), ("labels", C.c_void_p),
        ("num_fields", C.c_uint32), ("fp8_scale", C.c_void_p),
    ]


class SearchParams(C.Structure):
    _fields_ = [
        ("k", C.c_uint32), ("beam_width", C.c_uint32), ("rerank_size", C.c_uint32),
        ("use_codes", C.c_int32), ("filter", C.c_void_p), ("filter_nops", C.c_uint32),
        ("filter_pool", C.c_void_p),
    ]


class Spfresh(C.Structure):
    _fields_ = [
        ("d", C.c_uint32), ("metric", C.c_int32), ("num_blocks", C.c_uint32),
        ("block_cap", C.c_uint32), ("block_live", C.c_void_p), ("centroids", C.c_void_p),
        ("block_len", C.c_void_p), ("entry_ids", C.c_void_p), ("entry_codes", C.c_void_p),
        ("code_size", C.c_uint32), ("deleted", C.c_void_p), ("next_id", C.c_uint64),
        ("raw", C.c_void_p), ("quant", C.c_int32), ("pq_M", C.c_uint32), ("pq_K", C.c_uint32),
        ("pq_codebooks", C.c_void_p), ("int8_scale", C.c_float), ("int8_offset", C.c_float),
        ("rq_padded", C.c_uint32), ("rq_signs", C.c_void_p), ("probe_ratio", C.c_float),
        ("rerank_size", C.c_uint32),
    ]


def _declare(L):
    vp, u32, u64, i32, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_float
    sig = {
        "dgo_distance": (f32, [i32, vp, vp, u32]),
        "dgo_rand": (u64, [u64, u64, u64, u64]),
        "dgo_medoid": (u32, [vp, u64, u32, i32]),
        "dgo_robust_prune": (C.c_int, [u32, vp, vp, u32, vp, u32, i32, u32, f32, vp]),
        "dgo_build_vamana": (C.c_int, [vp, u64, u32, i32, u32, u32, f32, u64, u32, vp, i32]),
        "dgo_beam_search_table": (C.c_int, [vp, u32, vp, vp, vp, u32, u32, u32, i32, u32, u32, f32, vp, vp, vp]),
        "dgo_search_batch": (C.c_int, [vp, vp, vp, u32, vp, vp, vp, vp, vp, i32]),
        "dgo_incremental_search_batch": (C.c_int, [vp, vp, vp, u32, vp, u64, u64, vp, u32, vp, vp, vp, i32]),
        "dgo_filter_matches": (C.c_int, [vp, u32, vp, vp, u32]),
        "dgo_pq_encode": (None, [vp, u64, u32, u32, u32, vp, vp, i32]),
        "dgo_pq_lut": (None, [vp, u32, u32, u32, vp, vp]),
        "dgo_pq_adc": (f32, [vp, vp, u32, u32]),
        "dgo_int8_train": (None, [vp, u64, u32, vp, vp]),
        "dgo_int8_encode": (None, [vp, u64, u32, f32, f32, vp]),
        "dgo_int8_distance": (f32, [vp, vp, u32, f32]),
        "dgo_f16_encode": (None, [vp, u64, u32, vp]),
        "dgo_bf16_encode": (None, [vp, u64, u32, vp]),
        "dgo_fp8_encode": (None, [vp, u64, u32, vp, vp]),
        "dgo_e4m3_encode": (C.c_uint8, [C.c_float]),
        "dgo_e4m3_decode": (C.c_float, [C.c_uint8]),
        "dgo_f16_distance": (f32, [vp, vp, u32]),
        "dgo_rabitq_padded": (u32, [u32]),
        "dgo_rabitq_encode": (None, [vp, u64, u32, u32, vp, vp, vp]),
        "dgo_rabitq_query": (None, [vp, u32, u32, vp, vp, vp, vp]),
        "dgo_rabitq_distance": (f32, [vp, vp, vp, u32]),
        "dgo_rabitq_distance_with_bound": (None, [vp, vp, vp, u32, vp, vp]),
        "dgo_rabitq_decode": (None, [vp, u32, u32, vp, vp, vp]),
        "dgo_spfresh_search_batch": (C.c_int, [vp, vp, u32, u32, u32, vp, vp, vp, i32]),
        "dgo_exact_knn": (None, [vp, u64, u32, vp, u32, u32, i32, vp, vp, i32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ------------------------------------------------------------------ helpers
def distance(metric, a, b):
    a, b = _f32(a), _f32(b)
    return float(lib().dgo_distance(metric, _p(a), _p(b), a.shape[-1]))


def rand(seed, a, b, c):
    return int(lib().dgo_rand(seed, a, b, c))


def medoid(X, metric=L2SQ):
    X = _f32(X)
    return int(lib().dgo_medoid(_p(X), X.shape[0], X.shape[1], metric))


def robust_prune(node, ids, dists, X, R, alpha, metric=L2SQ):
    X = _f32(X)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    dists = _f32(dists)
    out = np.zeros(max(R, 1), dtype=np.uint32)
    n = lib().dgo_robust_prune(node, _p(ids), _p(dists), len(ids), _p(X), X.shape[1], metric, R,
                               alpha, _p(out))
    return out[:n].tolist()


def build_vamana(X, R, L_build, alpha=1.2, seed=0, metric=L2SQ, medoid_id=None, threads=0):
    X = _f32(X)
    if medoid_id is None:
        medoid_id = medoid(X, metric)
    adj = np.empty((X.shape[0], R), dtype=np.uint32)
    rc = lib().dgo_build_vamana(_p(X), X.shape[0], X.shape[1], metric, R, L_build, alpha, seed,
                                medoid_id, _p(adj), threads)
    if rc != 0:
        raise RuntimeError("oracle build failed")
    return adj, medoid_id


def beam_search_table(adj, node_dist, seeds, L, k, allow=None, filtered=False, expanded=0,
                      max_iter=0, early=float("inf")):
    adj = np.ascontiguousarray(adj, dtype=np.uint32)
    nd = _f32(node_dist)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
    al = None if allow is None else np.ascontiguousarray(allow, dtype=np.uint8)
    cap = max(k, 1) if filtered else max(k, 1)
    ids = np.zeros(cap, dtype=np.uint32)
    ds = np.zeros(cap, dtype=np.float32)
    n = C.c_uint32(0)
    lib().dgo_beam_search_table(_p(adj), adj.shape[1], _p(nd), _p(al), _p(seeds), len(seeds), L, k,
                                int(filtered), expanded, max_iter, early, _p(ids), _p(ds), C.byref(n))
    return list(zip(ids[: n.value].tolist(), ds[: n.value].tolist()))


def filter_program(ops, pool=()):
    """ops: list of (op, field, a, b) tuples in postfix order."""
    arr = (FilterOp * max(len(ops), 1))()
    for i, (op, field, a, b) in enumerate(ops):
        arr[i] = FilterOp(op, field, a, b)
    pool = np.ascontiguousarray(np.asarray(pool, dtype=np.uint64).reshape(-1))
    return arr, len(ops), pool


def filter_matches(ops, pool, labels):
    arr, n, pool = filter_program(ops, pool)
    lab = np.ascontiguousarray(labels, dtype=np.uint64)
    return bool(lib().dgo_filter_matches(arr, n, _p(pool), _p(lab), len(lab)))


class OracleIndex:
    """Holds numpy buffers alive for a DgoIndex view."""

    def __init__(self, vectors, adjacency, medoid_id, metric=L2SQ, native=False):
        self._L = lib_native() if native else lib()
        self.vectors = _f32(vectors)
        self.adj = np.ascontiguousarray(adjacency, dtype=np.uint32)
        self.s = Index()
        self.s.n, self.s.d = self.vectors.shape
        self.s.R = self.adj.shape[1]
        self.s.medoid = medoid_id
        self.s.metric = metric
        self.s.vectors = _p(self.vectors)
        self.s.adjacency = _p(self.adj)
        self.s.quant = Q_NONE
        self._keep = []

    def set_pq(self, codebooks, codes):
        cb = _f32(codebooks)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self._keep += [cb, codes]
        M, K, _ = cb.shape
        self.s.quant, self.s.pq_M, self.s.pq_K = Q_PQ, M, K
        self.s.pq_codebooks, self.s.codes, self.s.code_size = _p(cb), _p(codes), M

    def set_int8(self, scale, offset, codes):
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self._keep.append(codes)
        self.s.quant, self.s.int8_scale, self.s.int8_offset = Q_INT8, scale, offset
        self.s.codes, self.s.code_size = _p(codes), codes.shape[1]

    def set_f16(self, codes):
        codes = np.ascontiguousarray(codes, dtype=np.uint16)
        self._keep.append(codes)
        self.s.quant, self.s.codes, self.s.code_size = Q_F16, _p(codes), codes.shape[1] * 2

    def set_bf16(self, codes=None):
        """BF16 rows (bf16_encode of the vectors unless given) for the BF16
        traversal: search(..., use_codes=True, rerank=...)."""
        codes = bf16_encode(self.vectors) if codes is None else np.ascontiguousarray(codes, dtype=np.uint16)
        self._keep.append(codes)
        self.s.quant, self.s.codes, self.s.code_size = Q_BF16, _p(codes), codes.shape[1] * 2

    def set_fp8(self, codes, scales):
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        sc = _f32(scales)
        self._keep += [codes, sc]
        self.s.quant, self.s.codes, self.s.code_size = Q_FP8, _p(codes), codes.shape[1]
        self.s.fp8_scale = _p(sc)

    def set_rabitq(self, padded, centroid, signs, codes):
        cen, sg = _f32(centroid), _f32(signs)
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self._keep += [cen, sg, codes]
        self.s.quant, self.s.rq_padded = Q_RABITQ, padded
        self.s.rq_centroid, self.s.rq_signs = _p(cen), _p(sg)
        self.s.codes, self.s.code_size = _p(codes), codes.shape[1]

    def set_labels(self, labels):
        lab = np.ascontiguousarray(labels, dtype=np.uint64)
        self._keep.append(lab)
        self.s.labels, self.s.num_fields = _p(lab), lab.shape[1]

    def search(self, Q, k, L, rerank=0, use_codes=False, filter_ops=None, filter_pool=(),
               per_query_L=None, threads=0, with_stats=False):
        Q = _f32(Q).reshape(-1, self.s.d)
        nq = Q.shape[0]
        p = SearchParams()
        p.k, p.beam_width, p.rerank_size, p.use_codes = k, L, rerank, int(use_codes)
        keep = []
        if filter_ops:
            arr, n, pool = filter_program(filter_ops, filter_pool)
            keep += [arr, pool]
            p.filter, p.filter_nops, p.filter_pool = C.cast(arr, C.c_void_p), n, _p(pool)
        ids = np.zeros((nq, k), dtype=np.uint32)
        ds = np.zeros((nq, k), dtype=np.float32)
        cnt = np.zeros(nq, dtype=np.uint32)
        st = np.zeros((nq, 2), dtype=np.uint32)
        pl = None if per_query_L is None else np.ascontiguousarray(per_query_L, dtype=np.uint32)
        self._L.dgo_search_batch(C.byref(self.s), C.byref(p), _p(Q), nq, _p(pl), _p(ids), _p(ds),
                               _p(cnt), _p(st), threads)
        if with_stats:
            return ids, ds, cnt, st
        return ids, ds, cnt

    def incremental_search(self, Q, k, L, seeds, dead=None, ntomb=0, filter_ops=None, filter_pool=(),
                           threads=0, use_codes=False, rerank=0, code_limit=None):
        """IncrementalDiskANN search over this unified view (base rows, then delta
        rows): `seeds` entry points, `dead` a bool per row, `ntomb` the tombstone
        count; with use_codes, rows below code_limit are scored by their codes."""
        Q = _f32(Q).reshape(-1, self.s.d)
        nq = Q.shape[0]
        p = SearchParams()
        p.k, p.beam_width, p.use_codes, p.rerank_size = k, L, int(use_codes), rerank
        keep = []
        if filter_ops:
            arr, n, pool = filter_program(filter_ops, filter_pool)
            keep += [arr, pool]
            p.filter, p.filter_nops, p.filter_pool = C.cast(arr, C.c_void_p), n, _p(pool)
        sd = np.ascontiguousarray(seeds, dtype=np.uint32)
        dd = None if dead is None else np.ascontiguousarray(dead, dtype=np.uint8)
        ids = np.zeros((nq, k), dtype=np.uint32)
        ds = np.zeros((nq, k), dtype=np.float32)
        cnt = np.zeros(nq, dtype=np.uint32)
        cl = self.s.n if code_limit is None else code_limit
        self._L.dgo_incremental_search_batch(C.byref(self.s), C.byref(p), _p(sd), len(sd), _p(dd), int(ntomb),
                                           int(cl), _p(Q), nq, _p(ids), _p(ds), _p(cnt), threads)
        return ids, ds, cnt


def pq_encode(X, codebooks, threads=0):
    X, cb = _f32(X), _f32(codebooks)
    M, K, _ = cb.shape
    codes = np.empty((X.shape[0], M), dtype=np.uint8)
    lib().dgo_pq_encode(_p(X), X.shape[0], X.shape[1], M, K, _p(cb), _p(codes), threads)
    return codes


def pq_lut(q, codebooks):
    q, cb = _f32(q), _f32(codebooks)
    M, K, _ = cb.shape
    lut = np.empty((M, K), dtype=np.float32)
    lib().dgo_pq_lut(_p(q), q.shape[0], M, K, _p(cb), _p(lut))
    return lut


def pq_adc(lut, code):
    lut = _f32(lut)
    code = np.ascontiguousarray(code, dtype=np.uint8)
    return float(lib().dgo_pq_adc(_p(lut), _p(code), lut.shape[0], lut.shape[1]))


def int8_train(X):
    X = _f32(X)
    s, o = C.c_float(), C.c_float()
    lib().dgo_int8_train(_p(X), X.shape[0], X.shape[1], C.byref(s), C.byref(o))
    return s.value, o.value


def int8_encode(X, scale, offset):
    X = _f32(X).reshape(-1, np.shape(X)[-1])
    codes = np.empty(X.shape, dtype=np.uint8)
    lib().dgo_int8_encode(_p(X), X.shape[0], X.shape[1], scale, offset, _p(codes))
    return codes


def int8_distance(qc, cc, scale):
    qc = np.ascontiguousarray(qc, dtype=np.uint8)
    cc = np.ascontiguousarray(cc, dtype=np.uint8)
    return float(lib().dgo_int8_distance(_p(qc), _p(cc), len(qc), scale))


def f16_encode(X):
    X = _f32(X)
    out = np.empty(X.shape, dtype=np.uint16)
    lib().dgo_f16_encode(_p(X), X.size // X.shape[-1], X.shape[-1], _p(out))
    return out


def bf16_encode(X):
    """f32 -> BF16 bits (u16), rounded to nearest even."""
    X = _f32(X)
    out = np.empty(X.shape, dtype=np.uint16)
    lib().dgo_bf16_encode(_p(X), X.size // X.shape[-1], X.shape[-1], _p(out))
    return out


def fp8_encode(X):
    """(codes u8[n, d] e4m3, scales f32[n]) of the FP8 traversal copy."""
    X = _f32(X)
    n, d = X.shape
    codes = np.empty((n, d), dtype=np.uint8)
    scales = np.empty(n, dtype=np.float32)
    lib().dgo_fp8_encode(_p(X), n, d, _p(codes), _p(scales))
    return codes, scales


def rabitq_padded(d):
    return int(lib().dgo_rabitq_padded(d))


def rabitq_encode(X, padded, centroid, signs):
    X, cen, sg = _f32(X), _f32(centroid), _f32(signs)
    codes = np.empty((X.shape[0], padded // 8 + 8), dtype=np.uint8)
    lib().dgo_rabitq_encode(_p(X), X.shape[0], X.shape[1], padded, _p(cen), _p(sg), _p(codes))
    return codes


def rabitq_query(q, padded, centroid, signs):
    q, cen, sg = _f32(q), _f32(centroid), _f32(signs)
    planes = np.zeros(4 * (padded // 64), dtype=np.uint64)
    k5 = np.zeros(5, dtype=np.float32)
    lib().dgo_rabitq_query(_p(q), q.shape[0], padded, _p(cen), _p(sg), _p(planes), _p(k5))
    return planes, k5


def rabitq_distance(planes, k5, code, padded, with_bound=False):
    code = np.ascontiguousarray(code, dtype=np.uint8)
    if not with_bound:
        return float(lib().dgo_rabitq_distance(_p(planes), _p(k5), _p(code), padded))
    e, r = C.c_float(), C.c_float()
    lib().dgo_rabitq_distance_with_bound(_p(planes), _p(k5), _p(code), padded, C.byref(e), C.byref(r))
    return e.value, r.value


def rabitq_decode(code, d, padded, centroid, signs):
    code = np.ascontiguousarray(code, dtype=np.uint8)
    cen, sg = _f32(centroid), _f32(signs)
    out = np.empty(d, dtype=np.float32)
    lib().dgo_rabitq_decode(_p(code), d, padded, _p(cen), _p(sg), _p(out))
    return out


def exact_knn(X, Q, k, metric=L2SQ, threads=0):
    X, Q = _f32(X), _f32(Q).reshape(-1, np.shape(X)[1])
    ids = np.empty((Q.shape[0], k), dtype=np.uint32)
    ds = np.empty((Q.shape[0], k), dtype=np.float64)
    lib().dgo_exact_knn(_p(X), X.shape[0], X.shape[1], _p(Q), Q.shape[0], k, metric, _p(ids),
                        _p(ds), threads)
    return ids, ds


def spfresh_search(view: Spfresh, Q, k, nprobe, threads=0):
    Q = _f32(Q).reshape(-1, view.d)
    nq = Q.shape[0]
    ids = np.zeros((nq, k), dtype=np.uint64)
    ds = np.zeros((nq, k), dtype=np.float32)
    cnt = np.zeros(nq, dtype=np.uint32)
    lib().dgo_spfresh_search_batch(C.byref(view), _p(Q), nq, k, nprobe, _p(ids), _p(ds), _p(cnt),
                                   threads)
    return ids, ds, cnt


def _draw(seed, a, b, c, n):
    """floor(rand * n / 2^64): a uniform draw in [0, n) from the shared stream."""
    return (rand(seed, a, b, c) * n) >> 64


def pq_train(X, M, K, iterations, sample, seed):
    """ProductQuantizer::train (src/pq.rs:51-119, 290-410) with the product's
    seeded draws instead of thread_rng: a training sample of `sample` distinct
    rows by a partial Fisher-Yates shuffle (stream 0x7371), per subspace
    k-means++ seeding -- first centre from stream 0x6b6c, then D^2-weighted
    draws (stream 0x6b6d; an all-zero weight draws uniformly from 0x6b6e) --
    then `iterations` Lloyd steps: each row to its nearest centre (squared L2
    summed in coordinate order in f32, the first centre on ties), each centre
    to the f64 mean of its rows rounded to f32, an empty centre to a row drawn
    from stream 0x6b6f + iteration.  Codebooks f32[M, K, d/M]."""
    X = _f32(X)
    n, d = X.shape
    ds = d // M
    if sample > 0 and n > sample:
        perm = list(range(n))
        for i in range(sample):
            j = i + _draw(seed, 0x7371, i, 0, n - i)
            perm[i], perm[j] = perm[j], perm[i]
        rows = perm[:sample]
    else:
        rows = list(range(n))
    S = X[rows]
    ns = len(S)
    cb = np.zeros((M, K, ds), dtype=np.float32)

    def sqdist(x, c):  # x [r, ds], c [k, ds] -> f32 [r, k], sequential over ds
        acc = np.zeros((x.shape[0], c.shape[0]), dtype=np.float32)
        for j in range(ds):
            t = (x[:, j:j + 1] - c[None, :, j]).astype(np.float32)
            acc = (acc + (t * t).astype(np.float32)).astype(np.float32)
        return acc

    keff = min(K, ns)
    for m in range(M):
        Sm = S[:, m * ds:(m + 1) * ds]
        cb[m, 0] = Sm[_draw(seed, 0x6b6c, m, 0, ns)]
        mind = np.full(ns, np.float32(3.402823466e38), dtype=np.float32)
        for c in range(1, keff):
            mind = np.minimum(mind, sqdist(Sm, cb[m, c - 1:c])[:, 0])
            tot = float(np.sum(mind.astype(np.float64)))
            if tot <= 0.0:
                chosen = _draw(seed, 0x6b6e, m, c, ns)
            else:
                u = (rand(seed, 0x6b6d, m, c) >> 11) * (1.0 / 9007199254740992.0)
                cum = np.cumsum(mind.astype(np.float64))
                hit = np.nonzero(cum >= u * tot)[0]
                chosen = int(hit[0]) if len(hit) else ns - 1
            cb[m, c] = Sm[chosen]
        for c in range(keff, K):
            cb[m, c] = cb[m, c % keff]
    for it in range(iterations):
        for m in range(M):
            Sm = S[:, m * ds:(m + 1) * ds]
            a = np.argmin(sqdist(Sm, cb[m]), axis=1)
            new = cb[m].copy()
            for c in range(K):
                sel = Sm[a == c]
                if len(sel):
                    new[c] = (sel.astype(np.float64).sum(0) / len(sel)).astype(np.float32)
                else:
                    new[c] = Sm[_draw(seed, 0x6b6f + it, m, c, ns)]
            cb[m] = new
    return cb
