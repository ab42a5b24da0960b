"""pydiskann_b200 -- the pydiskann search surface on one NVIDIA B200.

Class and method names, defaults and error types follow the reference Python
binding (pydiskann 0.5.5, python/src/lib.rs):
  * ``metric="l2"`` is squared L2, ``"cosine"`` is 1 - cos, ``"dot"`` is 1 - a.b;
  * ``search`` returns ids, ``search_with_dists`` (id, distance) pairs,
    ``search_batch`` one id list per query;
  * bad metric / quantizer names raise ValueError, library errors
    RuntimeError, out-of-range ids IndexError.
Every search runs in libdgann.so (hand-written sm_100a kernels); there is no
CPU path.  Index construction (Vamana graph, PQ codebooks, codes) also runs
on the GPU.  Indexes persist in the reference's own file formats
(pydiskann_b200/formats.py): ``build(path=...)`` writes the DANN core file
(and, for FilteredDiskANN, ``{path}.idx`` / ``{path}.labels``), ``open`` /
``from_bytes`` load files and buffers the reference wrote, ``to_bytes`` and
``save_quantized`` write what the reference loads.

Batched array entry points (``search_arrays``) take numpy arrays or CUDA
tensors and return arrays, for callers that keep queries and results in HBM.
"""
from __future__ import annotations

import ctypes as C
import math
import warnings
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from . import formats as _fmt
from ._lib import PAD, DgError, check, lib, ptr  # noqa: F401  (DgError is public)

__all__ = [
    "DiskANN", "QuantizedDiskANN", "FilteredDiskANN", "IncrementalDiskANN", "SPFresh", "Filter", "build_graph",
    "medoid",
    "pq_train", "pq_encode", "exact_knn", "read_fvecs", "write_fvecs", "read_ivecs", "read_bvecs_as_f32",
    "simd_info",
]

_METRICS = {"l2": _lib.L2SQ, "cosine": _lib.COSINE, "dot": _lib.DOT, "euclidean": _lib.L2}


def _metric(m: str) -> int:
    try:
        return _METRICS[m]
    except KeyError:
        raise ValueError(f"unknown metric: {m}") from None


def _check_recorded_metric(meta, metric):
    """open_index_with / from_bytes (src/lib.rs:558-564, 583-589): the caller's metric
    is used; a different recorded distance only warns."""
    want = _fmt.DISTANCE_NAMES[metric]
    if meta.distance_name != want:
        warnings.warn(f"index recorded distance `{meta.distance_name}` but you opened with `{want}`",
                      RuntimeWarning, stacklevel=3)


def _f32(x, dim=None) -> np.ndarray:
    try:
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    except ValueError:
        # rows of different lengths: the reference's check (src/lib.rs:416-424)
        rows = list(x)
        d0 = len(rows[0])
        for i, r in enumerate(rows):
            if len(r) != d0:
                raise RuntimeError(f"Index error: Vector {i} has dimension {len(r)} but expected {d0}") from None
        raise
    if a.ndim == 1 and dim is not None:
        a = a.reshape(1, -1)
    return a


# ---------------------------------------------------------------- builders
def medoid(vectors, metric: str = "l2", device: int = 0) -> int:
    """calculate_medoid (src/lib.rs:748-768) on the GPU."""
    X = _f32(vectors)
    out = C.c_uint32()
    B = _lib.builder()
    check(B.dg_medoid(ptr(X), X.shape[0], X.shape[1], _metric(metric), device, C.byref(out)), B)
    return out.value


def build_graph(vectors, max_degree=64, build_beam_width=128, alpha=1.2, metric="l2", seed=0,
                medoid_id=None, device=0):
    """build_vamana_graph (src/lib.rs:774-917) on the GPU -> (adjacency u32[n,R], medoid)."""
    X = _f32(vectors)
    if X.ndim != 2 or X.shape[0] == 0:
        raise RuntimeError("Index error: No vectors provided")
    m = _metric(metric)
    if medoid_id is None:
        medoid_id = medoid(X, metric, device)
    adj = np.empty((X.shape[0], max_degree), dtype=np.uint32)
    B = _lib.builder()
    check(B.dg_build_vamana(ptr(X), X.shape[0], X.shape[1], m, max_degree, build_beam_width,
                            float(alpha), seed, medoid_id, device, ptr(adj)), B)
    return adj, medoid_id


def pq_train(vectors, num_subspaces=8, num_centroids=256, kmeans_iterations=20,
             training_sample_size=50_000, seed=0, device=0) -> np.ndarray:
    """ProductQuantizer::train (src/pq.rs:51-119) -> codebooks f32[M, K, dim/M]."""
    X = _f32(vectors)
    M, K = num_subspaces, num_centroids
    if X.shape[0] == 0:
        raise RuntimeError("Index error: No vectors to train on")
    cb = np.empty((M, K, X.shape[1] // max(M, 1)), dtype=np.float32)
    B = _lib.builder()
    check(B.dg_pq_train(ptr(X), X.shape[0], X.shape[1], M, K, kmeans_iterations,
                        training_sample_size, seed, device, ptr(cb)), B)
    return cb


def pq_encode(vectors, codebooks, device=0) -> np.ndarray:
    """ProductQuantizer::encode (src/pq.rs:122-149) on the GPU -> u8[n, M]."""
    X = _f32(vectors)
    cb = _f32(codebooks)
    M, K, _ = cb.shape
    codes = np.empty((X.shape[0], M), dtype=np.uint8)
    B = _lib.builder()
    check(B.dg_pq_encode(ptr(X), X.shape[0], X.shape[1], M, K, ptr(cb), device, ptr(codes)), B)
    return codes


def rabitq_encode(vectors, centroid, signs, padded=None, device=0):
    """RaBitQ::encode_with (src/rabitq.rs:218-256) on the GPU: residual codes of
    the rows against `centroid` (u8[n, padded/8 + 8])."""
    X = _f32(vectors)
    n, d = X.shape
    P = padded or rabitq_padded(d)
    cen = np.ascontiguousarray(centroid, dtype=np.float32).reshape(-1)
    sg = np.ascontiguousarray(signs, dtype=np.float32).reshape(-1)
    codes = np.empty((n, P // 8 + 8), dtype=np.uint8)
    B = _lib.builder()
    check(B.dg_rabitq_encode(ptr(X), n, d, P, ptr(cen), ptr(sg), device, ptr(codes)), B)
    return codes


def fp8_encode(vectors, device=0):
    """(codes u8[n, d] e4m3, scales f32[n]) as the FP8 traversal stores them."""
    X = _f32(vectors)
    n, d = X.shape
    codes = np.empty((n, d), dtype=np.uint8)
    scales = np.empty(n, dtype=np.float32)
    B = _lib.builder()
    check(B.dg_fp8_encode(ptr(X), n, d, device, ptr(codes), ptr(scales)), B)
    return codes, scales


def exact_knn(vectors, queries, k=10, metric="l2", device=0):
    """Brute-force k nearest neighbours (FP64 accumulation) -> (ids, dists)."""
    X = _f32(vectors)
    Q = _lib.query_rows(queries, X.shape[1])
    ids = np.empty((Q.shape[0], k), dtype=np.uint32)
    ds = np.empty((Q.shape[0], k), dtype=np.float32)
    B = _lib.builder()
    check(B.dg_exact_knn(ptr(X), X.shape[0], X.shape[1], ptr(Q), Q.shape[0], k, _metric(metric),
                         device, ptr(ids), ptr(ds)), B)
    return ids, ds


# ------------------------------------------------------------------ filter
class Filter:
    """Filter predicate over a vector's label fields (src/filtered.rs:61-135).

    Compiled to the postfix DgFilterOp program the kernels evaluate.
    """

    __slots__ = ("_kind", "_args")

    def __init__(self, kind, args=()):
        self._kind = kind
        self._args = args

    @staticmethod
    def none():
        return Filter("none")

    @staticmethod
    def eq(field: int, value: int):
        return Filter("eq", (field, value))

    @staticmethod
    def in_(field: int, values: Iterable[int]):
        return Filter("in", (field, frozenset(int(v) for v in values)))

    @staticmethod
    def lt(field: int, value: int):
        return Filter("lt", (field, value))

    @staticmethod
    def gt(field: int, value: int):
        return Filter("gt", (field, value))

    @staticmethod
    def range(field: int, min: int, max: int):  # noqa: A002 - reference argument names
        return Filter("range", (field, min, max))

    @staticmethod
    def and_(filters: Sequence["Filter"]):
        return Filter("and", tuple(filters))

    @staticmethod
    def or_(filters: Sequence["Filter"]):
        return Filter("or", tuple(filters))

    def is_none(self) -> bool:
        return self._kind == "none"

    def matches(self, labels: Sequence[int]) -> bool:
        k, a = self._kind, self._args
        if k == "none":
            return True
        if k in ("and", "or"):
            res = (f.matches(labels) for f in a)
            return all(res) if k == "and" else any(res)
        field = a[0]
        if field >= len(labels):
            return False
        v = labels[field]
        if k == "eq":
            return v == a[1]
        if k == "in":
            return v in a[1]
        if k == "lt":
            return v < a[1]
        if k == "gt":
            return v > a[1]
        return a[1] <= v <= a[2]

    def compile(self, ops: list, pool: list):
        """Append this filter's postfix program to ops (FilterOp tuples)."""
        k, a = self._kind, self._args
        if k == "none":
            return
        if k in ("and", "or"):
            for f in a:
                if f.is_none():
                    ops.append((_lib.F_TRUE, 0, 0, 0))
                else:
                    f.compile(ops, pool)
            ops.append((_lib.F_AND if k == "and" else _lib.F_OR, len(a), 0, 0))
            return
        field = a[0]
        if k == "eq":
            ops.append((_lib.F_EQ, field, a[1], 0))
        elif k == "lt":
            ops.append((_lib.F_LT, field, a[1], 0))
        elif k == "gt":
            ops.append((_lib.F_GT, field, a[1], 0))
        elif k == "range":
            ops.append((_lib.F_RANGE, field, a[1], a[2]))
        else:
            vals = sorted(a[1])
            ops.append((_lib.F_IN, field, len(pool), len(vals)))
            pool.extend(vals)

    def program(self):
        ops, pool = [], []
        self.compile(ops, pool)
        return ops, pool

    def __repr__(self):
        return f"Filter.{self._kind}{self._args!r}"


class PackedFilters:
    """Per-query filter programs compiled once, for repeated batched searches
    (``search_arrays(..., filters=pack_filters(list_of_filters))``)."""

    def __init__(self, filters):
        self.n = len(filters)
        self.arr, self.offs, self.pool, self.plen = _pack_programs([f.program() for f in filters])


def pack_filters(filters):
    return PackedFilters(list(filters))


def _pack_programs(progs):
    """[(ops, pool)] per query -> (FilterOp array, offsets u32[nq+1], pool u64)."""
    all_ops, offs, pool = [], [0], []
    for ops, p in progs:
        base = len(pool)
        for (op, field, a, b) in ops:
            if op == _lib.F_IN:
                a += base
            all_ops.append((op, field, a, b))
        pool.extend(p)
        offs.append(len(all_ops))
    arr = (_lib.FilterOp * max(len(all_ops), 1))()
    for i, (op, field, a, b) in enumerate(all_ops):
        arr[i] = _lib.FilterOp(op, field, a, b)
    return arr, np.asarray(offs, dtype=np.uint32), np.asarray(pool if pool else [0], dtype=np.uint64), len(pool)


def _check_out(out, nq, k, dev):
    """Caller-given result buffers (ids, dists, counts): the library writes
    nq * k ids and distances and nq counts of 4 bytes each, contiguously,
    into device memory for CUDA queries and host memory otherwise."""
    for a, need, name in zip(out, (nq * k, nq * k, nq), ("ids", "dists", "counts")):
        tensor = hasattr(a, "data_ptr")
        size = a.numel() if tensor else np.asarray(a).size
        item = a.element_size() if tensor else a.itemsize
        contiguous = a.is_contiguous() if tensor else a.flags.c_contiguous
        on_device = tensor and getattr(a, "is_cuda", False)
        if size < need or item != 4 or not contiguous or on_device != dev or (not tensor and not a.flags.writeable):
            raise ValueError(f"out[{name}] must be a writable contiguous {'CUDA' if dev else 'host'} array of "
                             f">= {need} 4-byte elements")


# ------------------------------------------------------------------- index
class _Index:
    """A device-resident graph index (one libdgann DgIndex handle)."""

    def __init__(self, vectors, adjacency, medoid_id, metric="l2", device=0, hbm_budget_bytes=0):
        X = _f32(vectors)
        adj = np.ascontiguousarray(adjacency, dtype=np.uint32)
        if X.ndim != 2 or X.shape[0] == 0:
            raise RuntimeError("Index error: No vectors provided")
        self._X = X
        self._metric_name = metric
        self._metric = _metric(metric)
        self.device = device
        d = _lib.IndexDesc()
        d.dim, d.max_degree, d.num_vectors = X.shape[1], adj.shape[1], X.shape[0]
        d.medoid, d.metric = int(medoid_id), self._metric
        d.vectors, d.adjacency = ptr(X), ptr(adj)
        d.device, d.hbm_budget_bytes = device, hbm_budget_bytes
        h = C.c_void_p()
        check(lib().dg_index_create(C.byref(d), C.byref(h)))
        self._h = h
        self.adjacency = adj
        self.medoid_id = int(medoid_id)
        self._bf16 = False
        self._quant = None

    def close(self):
        if getattr(self, "_h", None):
            lib().dg_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- properties
    @property
    def num_vectors(self) -> int:
        return self._X.shape[0]

    @property
    def dim(self) -> int:
        return self._X.shape[1]

    @property
    def max_degree(self) -> int:
        return self.adjacency.shape[1]

    def get_vector(self, id: int):  # noqa: A002
        if id < 0 or id >= self.num_vectors:
            raise IndexError(id)
        return self._X[id].tolist()

    def to_bytes(self) -> bytes:
        """DiskANN::to_bytes (src/lib.rs:630-632): the DANN core file's bytes."""
        return _fmt.core_bytes(self._X, self.adjacency, self.medoid_id, self._metric_name)

    def enable_bf16(self):
        if not self._bf16:
            check(lib().dg_index_enable_bf16(self._h))
            self._bf16 = True

    def enable_fp8(self):
        """FP8 (e4m3, per-vector scales) copy for ``traversal=TRAVERSE_FP8``; follow
        it with an FP32 rerank (``rerank_size``).  No counterpart in the reference."""
        if not getattr(self, "_fp8", False):
            check(lib().dg_index_enable_fp8(self._h))
            self._fp8 = True

    # -- the batched entry point
    def _params(self, queries, k, beam_width, traversal, rerank_size, filters, per_query_beam, out, stream,
                with_stats, per_query_k=None):
        """DgSearchParams and buffers of one batched call (see search_arrays)."""
        dev = hasattr(queries, "data_ptr") and getattr(queries, "is_cuda", False)
        p = _lib.SearchParams()
        p.k, p.beam_width, p.rerank_size, p.traversal = k, beam_width, rerank_size, traversal
        keep = []
        if dev:
            import torch

            Q = queries.contiguous()
            if Q.dim() == 1:
                Q = Q.reshape(1, -1)
            if Q.dim() != 2:
                raise ValueError(f"queries must be one query or a 2-D batch, not shape {tuple(Q.shape)}")
            if Q.shape[1] != self.dim:
                raise ValueError(f"Query dim {Q.shape[1]} != index dim {self.dim}")
            if Q.dtype != torch.float32:
                raise ValueError(f"CUDA queries must be float32, not {Q.dtype}")
            nq = Q.shape[0]
            if out is None:
                out = (torch.empty((nq, k), dtype=torch.int32, device=Q.device),
                       torch.empty((nq, k), dtype=torch.float32, device=Q.device),
                       torch.empty((nq,), dtype=torch.int32, device=Q.device))
            stats = torch.empty((nq, 2), dtype=torch.int32, device=Q.device) if with_stats else None
            # ordered on the caller's torch stream (handle 0 is the legacy default stream)
            p.flags = _lib.FLAG_DEVICE_PTRS | _lib.FLAG_STREAM
            p.stream = stream if stream is not None else torch.cuda.current_stream(Q.device).cuda_stream
        else:
            Q = _f32(queries)
            if Q.ndim == 1:
                Q = Q.reshape(1, -1)
            nq = Q.shape[0]
            if Q.shape[1] != self.dim:
                raise ValueError(f"Query dim {Q.shape[1]} != index dim {self.dim}")
            if out is None:
                out = (np.empty((nq, k), dtype=np.uint32), np.empty((nq, k), dtype=np.float32),
                       np.empty((nq,), dtype=np.uint32))
            stats = np.empty((nq, 2), dtype=np.uint32) if with_stats else None
            if stream is not None:
                p.flags = _lib.FLAG_STREAM
                p.stream = stream
        _check_out(out, nq, k, dev)
        if isinstance(filters, PackedFilters):
            if filters.n != nq:
                raise ValueError("one filter per query expected")
            p.filter_ops, p.filter_offsets = C.cast(filters.arr, C.c_void_p), ptr(filters.offs)
            p.filter_pool, p.filter_pool_len = ptr(filters.pool), filters.plen
        elif filters is not None:
            if isinstance(filters, Filter):
                if not filters.is_none():
                    arr, offs, pool, plen = _pack_programs([filters.program()])
                    keep += [arr, pool]
                    p.filter_ops, p.filter_nops = C.cast(arr, C.c_void_p), int(offs[-1])
                    p.filter_pool, p.filter_pool_len = ptr(pool), plen
            else:
                if len(filters) != nq:
                    raise ValueError("one filter per query expected")
                arr, offs, pool, plen = _pack_programs([f.program() for f in filters])
                keep += [arr, offs, pool]
                p.filter_ops, p.filter_offsets = C.cast(arr, C.c_void_p), ptr(offs)
                p.filter_pool, p.filter_pool_len = ptr(pool), plen
        if per_query_beam is not None:
            pl = np.ascontiguousarray(per_query_beam, dtype=np.uint32).reshape(-1)
            if len(pl) != nq:  # the library reads one beam width per query
                raise ValueError(f"one beam width per query expected: {len(pl)} for {nq} queries")
            keep.append(pl)
            p.per_query_beam = ptr(pl)
        if per_query_k is not None:
            pk = np.ascontiguousarray(per_query_k, dtype=np.uint32).reshape(-1)
            if len(pk) != nq:  # the library reads one k per query
                raise ValueError(f"one k per query expected: {len(pk)} for {nq} queries")
            keep.append(pk)
            p.per_query_k = ptr(pk)
        return p, Q, nq, out, stats, keep

    def search_arrays(self, queries, k=10, beam_width=128, traversal=_lib.TRAVERSE_F32,
                      rerank_size=0, filters=None, per_query_beam=None, out=None, stream=None,
                      with_stats=False, per_query_k=None):
        """Batched search over numpy arrays (host) or CUDA tensors (device).

        Returns (ids u32[nq,k], dists f32[nq,k], counts u32[nq]) of the same
        kind as `queries`; rows are padded with PAD / +inf past counts.
        `filters` is one Filter for all queries or a list of one per query;
        `per_query_k` (each in [1, k]) gives query i its own k in a row of k.
        """
        p, Q, nq, out, stats, keep = self._params(queries, k, beam_width, traversal, rerank_size, filters,
                                                  per_query_beam, out, stream, with_stats, per_query_k)
        check(lib().dg_search_batch(self._h, C.byref(p), ptr(Q), nq, ptr(out[0]), ptr(out[1]),
                                    ptr(out[2]), ptr(stats)))
        del keep
        if with_stats:
            return out[0], out[1], out[2], stats
        return out

    def autotune(self, queries, k=10, beam_width=128, traversal=_lib.TRAVERSE_F32, rerank_size=0, filters=None,
                 per_query_beam=None, reps=3):
        """Times this search (same arguments as search_arrays) under candidate
        launch schedules -- visited-table size, query order, CTAs per SM, warps
        per CTA -- and keeps the fastest for later searches of the same kind
        (dg_index_autotune).  Returns {"hbits", "order", "occ_pct",
        "warps_per_cta": the chosen schedule, "ms": {bits: ms per call of each
        table size}}."""
        p, Q, nq, _, _, keep = self._params(queries, k, beam_width, traversal, rerank_size, filters,
                                            per_query_beam, None, None, False)
        best = C.c_uint32()
        ms = (C.c_float * 6)()
        check(lib().dg_index_autotune(self._h, C.byref(p), ptr(Q), nq, reps, C.byref(best), ms))
        del keep
        hb, order, occ, wpb = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().dg_index_tuned_schedule(self._h, C.byref(hb), C.byref(order), C.byref(occ), C.byref(wpb)))
        return {"hbits": hb.value, "order": order.value, "occ_pct": occ.value, "warps_per_cta": wpb.value,
                "ms": {8 + i: round(ms[i], 4) for i in range(6) if ms[i] >= 0}}

    # -- reference-shaped helpers
    def _rows(self, ids, dists, cnt):
        return [[(int(ids[i, j]), float(dists[i, j])) for j in range(int(cnt[i]))] for i in range(len(cnt))]


class DiskANN(_Index):
    """DiskANN<D> (src/lib.rs) search surface: plain FP32 Vamana beam search.

    ``traversal="bf16"`` reads a BF16 copy of the vectors during the beam
    search (FP32 accumulation) and ``rerank_size`` then re-scores the best
    candidates with the FP32 rows.
    """

    @staticmethod
    def build(vectors, path=None, metric="l2", max_degree=64, build_beam_width=128, alpha=1.2,
              seed=0, device=0):
        X = _f32(vectors)
        if X.ndim != 2 or X.shape[0] == 0:
            raise RuntimeError("Index error: No vectors provided")
        adj, med = build_graph(X, max_degree, build_beam_width, alpha, metric, seed, None, device)
        if path is not None:  # build_index_with_params writes the core file (src/lib.rs:355-505)
            _fmt.write_core(path, X, adj, med, metric)
        return DiskANN(X, adj, med, metric, device)

    @staticmethod
    def from_graph(vectors, adjacency, medoid_id, metric="l2", device=0, hbm_budget_bytes=0):
        return DiskANN(vectors, adjacency, medoid_id, metric, device, hbm_budget_bytes)

    @staticmethod
    def open(path, metric="l2", device=0, hbm_budget_bytes=0):
        """DiskANN::open_index_with (src/lib.rs:507-577): a DANN core file."""
        _metric(metric)
        m, X, A = _fmt.read_core(path)
        _check_recorded_metric(m, metric)
        return DiskANN(X, A, m.medoid_id, metric, device, hbm_budget_bytes)

    @staticmethod
    def from_bytes(data, metric="l2", device=0, hbm_budget_bytes=0):
        """DiskANN::from_bytes (src/lib.rs:580-601): a core file's bytes."""
        _metric(metric)
        m, X, A = _fmt.parse_core(data)
        _check_recorded_metric(m, metric)
        return DiskANN(X, A, m.medoid_id, metric, device, hbm_budget_bytes)

    def search_with_dists(self, query, k=10, beam_width=128):
        ids, ds, cnt = self.search_arrays(_f32(query).reshape(1, -1), k, beam_width)
        return self._rows(ids, ds, cnt)[0]

    def search(self, query, k=10, beam_width=128):
        return [i for i, _ in self.search_with_dists(query, k, beam_width)]

    def search_batch(self, queries, k=10, beam_width=128):
        ids, ds, cnt = self.search_arrays(_lib.query_rows(queries, self.dim), k, beam_width)
        return [ids[i, : cnt[i]].astype(np.int64).tolist() for i in range(len(cnt))]


class QuantizedDiskANN(_Index):
    """QuantizedDiskANN<D> (src/quantized.rs): beam search on codes + exact rerank."""

    def __init__(self, vectors, adjacency, medoid_id, metric="l2", device=0, rerank_size=0,
                 hbm_budget_bytes=0):
        super().__init__(vectors, adjacency, medoid_id, metric, device, hbm_budget_bytes)
        self.rerank_size = rerank_size

    @staticmethod
    def build(vectors, path=None, quantizer="f16", metric="l2", rerank_size=0, pq_subspaces=8,
              max_degree=64, build_beam_width=128, alpha=1.2, seed=0, device=0):
        if quantizer not in ("f16", "int8", "pq", "rabitq"):
            raise ValueError(f"unknown quantizer: {quantizer}")
        _metric(metric)
        X = _f32(vectors)
        if X.ndim != 2 or X.shape[0] == 0:
            raise RuntimeError("Index error: No vectors provided")
        adj, med = build_graph(X, max_degree, build_beam_width, alpha, metric, seed, None, device)
        if path is not None:  # build_* writes the base core file (src/quantized.rs:584-634)
            _fmt.write_core(path, X, adj, med, metric)
        q = QuantizedDiskANN(X, adj, med, metric, device, rerank_size)
        if quantizer == "f16":
            q.attach_f16()
        elif quantizer == "int8":
            q.attach_int8(*int8_params(X))
        elif quantizer == "pq":
            q.attach_pq(pq_train(X, pq_subspaces, 256, 20, 50_000, seed, device))
        else:
            cen, signs = rabitq_params(X, seed)
            q.attach_rabitq(cen, signs)
        return q

    def attach_pq(self, codebooks, codes=None):
        cb = _f32(codebooks)
        M, K, ds = cb.shape
        if ds * M != self.dim:
            raise RuntimeError(f"Index error: Dimension {self.dim} not divisible by num_subspaces {M}")
        c = None if codes is None else np.ascontiguousarray(codes, dtype=np.uint8)
        check(lib().dg_index_attach_pq(self._h, M, K, ptr(cb), ptr(c)))
        self._quant = ("pq", cb)

    def attach_int8(self, scale, offset, codes=None):
        c = None if codes is None else np.ascontiguousarray(codes, dtype=np.uint8)
        check(lib().dg_index_attach_int8(self._h, float(scale), float(offset), ptr(c)))
        self._quant = ("int8", (scale, offset))

    def attach_f16(self, codes=None):
        """codes: u16[n, dim] f16 bit patterns (a QANN sidecar's); None encodes on the GPU."""
        c = None
        if codes is not None:
            c = np.ascontiguousarray(codes).view(np.uint8).reshape(self.num_vectors, -1)
            if c.shape[1] != 2 * self.dim:
                raise ValueError(f"F16 codes must be {2 * self.dim} bytes per vector")
        check(lib().dg_index_attach_f16_codes(self._h, ptr(c)))
        self._quant = ("f16", None)

    def attach_rabitq(self, centroid, signs, codes=None):
        cen, sg = _f32(centroid), _f32(signs)
        padded = sg.size // 3
        c = None if codes is None else np.ascontiguousarray(codes, dtype=np.uint8)
        check(lib().dg_index_attach_rabitq(self._h, padded, ptr(cen), ptr(sg), ptr(c)))
        self._quant = ("rabitq", (cen, sg))

    # -- persistence: the QANN sidecar (src/quantized.rs:420-575)
    @staticmethod
    def open(base_path, quantized_path, metric="l2", rerank_size=0, device=0, hbm_budget_bytes=0):
        """QuantizedDiskANN::open (src/quantized.rs:444-454): a core file and its sidecar."""
        _metric(metric)
        m, X, A = _fmt.read_core(base_path)
        _check_recorded_metric(m, metric)
        state, codes = _fmt.read_sidecar(quantized_path, m.num_vectors)
        q = QuantizedDiskANN(X, A, m.medoid_id, metric, device, rerank_size, hbm_budget_bytes)
        q.attach_state(state, codes)
        return q

    @staticmethod
    def from_bytes(data, metric="l2", rerank_size=0, device=0, hbm_budget_bytes=0):
        """QuantizedDiskANN::from_bytes (src/quantized.rs:468-488): [base_len][core][sidecar]."""
        _metric(metric)
        base, rest = _fmt.split_prefixed(data)
        m, X, A = _fmt.parse_core(base)
        _check_recorded_metric(m, metric)
        state, codes = _fmt.parse_sidecar(rest, m.num_vectors)
        q = QuantizedDiskANN(X, A, m.medoid_id, metric, device, rerank_size, hbm_budget_bytes)
        q.attach_state(state, codes)
        return q

    def attach_state(self, state, codes=None):
        """Attaches a formats.QuantizerState (the sidecar's quantizer) and its codes."""
        if state.dim != self.dim:
            raise RuntimeError(f"Index error: quantizer dim {state.dim} != index dim {self.dim}")
        if state.kind == "pq":
            cb = state.codebooks.reshape(state.num_subspaces, state.num_centroids, state.subspace_dim)
            self.attach_pq(cb, codes)
        elif state.kind == "int8":
            self.attach_int8(state.scale, state.offset, codes)
        elif state.kind == "f16":
            self.attach_f16(codes)
        else:
            if state.padded != rabitq_padded(self.dim):
                raise RuntimeError(f"Index error: RaBitQ padded {state.padded} != {rabitq_padded(self.dim)}")
            self.attach_rabitq(state.centroid, state.signs, codes)

    def quantizer_state(self):
        """The attached quantizer as the sidecar's QuantizerState."""
        if self._quant is None:
            raise RuntimeError("Index error: no quantizer attached")
        kind, p = self._quant
        if kind == "pq":
            M, K, ds = p.shape
            return _fmt.QuantizerState("pq", self.dim, M, K, ds, codebooks=p.reshape(-1))
        if kind == "int8":
            return _fmt.QuantizerState("int8", self.dim, scale=p[0], offset=p[1])
        if kind == "f16":
            return _fmt.QuantizerState("f16", self.dim)
        cen, sg = p
        return _fmt.QuantizerState("rabitq", self.dim, padded=sg.size // 3, centroid=cen, signs=sg)

    def codes(self) -> np.ndarray:
        """The codes in HBM, u8[n, code_size] as the sidecar stores them."""
        cs = C.c_uint32()
        check(lib().dg_index_get_codes(self._h, None, 0, C.byref(cs)))
        out = np.empty((self.num_vectors, cs.value), np.uint8)
        check(lib().dg_index_get_codes(self._h, ptr(out), out.size, None))
        return out

    def save_quantized(self, path):
        """QuantizedDiskANN::save_quantized (src/quantized.rs:435-441)."""
        _fmt.write_sidecar(path, self.quantizer_state(), self.codes())

    def to_bytes(self) -> bytes:
        """QuantizedDiskANN::to_bytes (src/quantized.rs:456-466)."""
        return _fmt.join_prefixed(super().to_bytes(), _fmt.sidecar_bytes(self.quantizer_state(), self.codes()))

    def search_arrays(self, queries, k=10, beam_width=128, traversal=_lib.TRAVERSE_CODES,
                      rerank_size=None, **kw):
        rr = self.rerank_size if rerank_size is None else rerank_size
        return super().search_arrays(queries, k, beam_width, traversal, rr, **kw)

    def autotune(self, queries, k=10, beam_width=128, traversal=_lib.TRAVERSE_CODES, rerank_size=None, **kw):
        rr = self.rerank_size if rerank_size is None else rerank_size
        return super().autotune(queries, k, beam_width, traversal, rr, **kw)

    def search_with_dists(self, query, k=10, beam_width=128):
        ids, ds, cnt = self.search_arrays(_f32(query).reshape(1, -1), k, beam_width)
        return self._rows(ids, ds, cnt)[0]

    def search(self, query, k=10, beam_width=128):
        return [i for i, _ in self.search_with_dists(query, k, beam_width)]

    def search_batch(self, queries, k=10, beam_width=128):
        ids, ds, cnt = self.search_arrays(_lib.query_rows(queries, self.dim), k, beam_width)
        return [ids[i, : cnt[i]].astype(np.int64).tolist() for i in range(len(cnt))]

    def search_filtered_with_dists(self, query, k, beam_width, labels, filter):  # noqa: A002
        """QuantizedDiskANN::search_filtered_with_dists (src/quantized.rs:350-398)."""
        if not getattr(self, "_labels_attached", False):
            self.attach_labels(labels)
        ids, ds, cnt = self.search_arrays(_f32(query).reshape(1, -1), k, beam_width, filters=filter)
        return self._rows(ids, ds, cnt)[0]

    def attach_labels(self, labels):
        lab = np.ascontiguousarray(labels, dtype=np.uint64)
        if lab.shape[0] != self.num_vectors:
            raise ValueError(f"Labels count {lab.shape[0]} != index vectors {self.num_vectors}")
        check(lib().dg_index_attach_labels(self._h, lab.shape[1], ptr(lab)))
        self._labels = lab
        self._labels_attached = True


class FilteredDiskANN(_Index):
    """FilteredDiskANN<D> (src/filtered.rs): label-filtered beam search."""

    def __init__(self, vectors, adjacency, medoid_id, labels, metric="l2", device=0,
                 hbm_budget_bytes=0):
        lab = np.ascontiguousarray(labels, dtype=np.uint64)
        X = _f32(vectors)
        if lab.ndim != 2 or lab.shape[0] != X.shape[0]:
            raise RuntimeError(
                f"Index error: vectors.len() ({X.shape[0]}) != labels.len() ({lab.shape[0] if lab.ndim else 0})")
        super().__init__(X, adjacency, medoid_id, metric, device, hbm_budget_bytes)
        check(lib().dg_index_attach_labels(self._h, lab.shape[1], ptr(lab)))
        self._labels = lab

    @staticmethod
    def build(vectors, labels, path=None, metric="l2", max_degree=64, build_beam_width=128,
              alpha=1.2, seed=0, device=0):
        lab = [list(map(int, l)) for l in labels]
        nf = len(lab[0]) if lab else 0
        for i, l in enumerate(lab):
            if len(l) != nf:
                raise RuntimeError(f"Index error: Label {i} has {len(l)} fields, expected {nf}")
        X = _f32(vectors)
        if len(lab) != X.shape[0]:
            raise RuntimeError(f"Index error: vectors.len() ({X.shape[0]}) != labels.len() ({len(lab)})")
        adj, med = build_graph(X, max_degree, build_beam_width, alpha, metric, seed, None, device)
        arr = np.asarray(lab, dtype=np.uint64).reshape(X.shape[0], nf)
        if path is not None:  # {path}.idx and {path}.labels (src/filtered.rs:202-208)
            _fmt.write_core(f"{path}.idx", X, adj, med, metric)
            _fmt.write_labels(f"{path}.labels", arr)
        return FilteredDiskANN(X, adj, med, arr, metric, device)

    @staticmethod
    def open(path, metric="l2", device=0, hbm_budget_bytes=0):
        """FilteredDiskANN::open (src/filtered.rs:219-241): `{path}.idx` and `{path}.labels`."""
        _metric(metric)
        m, X, A = _fmt.read_core(f"{path}.idx")
        _check_recorded_metric(m, metric)
        return FilteredDiskANN._with_labels(m, X, A, _fmt.read_labels(f"{path}.labels"), metric, device,
                                            hbm_budget_bytes)

    @staticmethod
    def from_bytes(data, metric="l2", device=0, hbm_budget_bytes=0):
        """FilteredDiskANN::from_bytes (src/filtered.rs:256-285): [index_len][core][labels]."""
        _metric(metric)
        base, rest = _fmt.split_prefixed(data, "index data")
        m, X, A = _fmt.parse_core(base)
        _check_recorded_metric(m, metric)
        return FilteredDiskANN._with_labels(m, X, A, _fmt.parse_labels(rest), metric, device, hbm_budget_bytes)

    @staticmethod
    def _with_labels(m, X, A, lab, metric, device, hbm_budget_bytes):
        if lab.shape[0] != m.num_vectors:
            raise RuntimeError(f"Index error: Labels count ({lab.shape[0]}) != index vectors ({m.num_vectors})")
        return FilteredDiskANN(X, A, m.medoid_id, lab, metric, device, hbm_budget_bytes)

    def to_bytes(self) -> bytes:
        """FilteredDiskANN::to_bytes (src/filtered.rs:245-254)."""
        return _fmt.join_prefixed(super().to_bytes(), _fmt.labels_bytes(self._labels))

    @property
    def num_fields(self) -> int:
        return self._labels.shape[1]

    def get_labels(self, id: int):  # noqa: A002
        if id < 0 or id >= self.num_vectors:
            return None
        return [int(v) for v in self._labels[id]]  # u64 values, as Vec<u64>

    def count_matching(self, filter: Filter) -> int:  # noqa: A002
        ops, pool = filter.program()
        arr, offs, pl, plen = _pack_programs([(ops, pool)])
        out = C.c_uint64()
        check(lib().dg_count_matching(self._h, C.cast(arr, C.c_void_p), len(ops), ptr(pl), plen,
                                      C.byref(out)))
        return out.value

    def search(self, query, k=10, beam_width=128):
        ids, ds, cnt = self.search_arrays(_f32(query).reshape(1, -1), k, beam_width)
        return ids[0, : cnt[0]].astype(np.int64).tolist()

    def search_filtered_with_dists(self, query, filter, k=10, beam_width=128):  # noqa: A002
        ids, ds, cnt = self.search_arrays(_f32(query).reshape(1, -1), k, beam_width, filters=filter)
        return self._rows(ids, ds, cnt)[0]

    def search_filtered(self, query, filter, k=10, beam_width=128):  # noqa: A002
        return [i for i, _ in self.search_filtered_with_dists(query, filter, k, beam_width)]

    def search_filtered_batch(self, queries, filter, k=10, beam_width=128):  # noqa: A002
        ids, ds, cnt = self.search_arrays(_lib.query_rows(queries, self.dim), k, beam_width,
                                          filters=filter)
        return [ids[i, : cnt[i]].astype(np.int64).tolist() for i in range(len(cnt))]


# --------------------------------------------------------- quantizer params
def int8_params(vectors):
    """Int8Quantizer::train (src/sq.rs:128-157): one global (scale, offset)."""
    X = _f32(vectors)
    lo, hi = np.float32(X.min()), np.float32(X.max())
    rng = np.float32(hi - lo)
    scale = np.float32(1.0) if abs(rng) < np.finfo(np.float32).eps else np.float32(rng / np.float32(255.0))
    return float(scale), float(lo)


def rabitq_padded(dim: int) -> int:
    """src/rabitq.rs:83: next_power_of_two(max(dim, 64))."""
    return 1 << max(6, math.ceil(math.log2(max(dim, 1))))


def rabitq_params(vectors, seed=0):
    """RaBitQ::train (src/rabitq.rs:78-107): centroid and 3 rounds of +-1/sqrt(padded) signs.

    The reference draws the signs from StdRng(0x7ab17); callers holding a
    trained reference quantizer pass its signs to attach_rabitq instead.
    """
    X = _f32(vectors)
    cen = (X.astype(np.float64).sum(axis=0) / X.shape[0]).astype(np.float32)
    P = rabitq_padded(X.shape[1])
    scale = np.float32(1.0) / np.float32(math.sqrt(P))
    bits = np.random.default_rng([seed, 0x7AB17]).integers(0, 2, size=3 * P)
    signs = np.where(bits == 1, scale, -scale).astype(np.float32)
    return cen, signs


# ----------------------------------------------------------------- formats
def _read_vecs(path, dtype):
    """Records of a little-endian u32 count followed by that many elements (the
    fvecs / ivecs / bvecs layout, src/formats.rs:7-113), as numpy arrays.
    Records may differ in length.  As with read_exact there, a trailing length
    field of 1-3 bytes ends the file, and a record cut short is an I/O error."""
    dt = np.dtype(dtype)
    try:
        buf = np.fromfile(path, dtype=np.uint8)
    except OSError as e:
        raise _fmt.io_error(e) from None
    n = buf.size
    if n >= 4:  # every record the same length: one reshape
        d = int(buf[:4].view("<u4")[0])
        rec = 4 + d * dt.itemsize
        if n % rec == 0:
            recs = buf.reshape(-1, rec)
            if np.all(np.ascontiguousarray(recs[:, :4]).view("<u4") == d):
                return list(np.ascontiguousarray(recs[:, 4:]).view(dt).reshape(len(recs), d))
    out, pos = [], 0
    while n - pos >= 4:
        d = int(buf[pos:pos + 4].view("<u4")[0])
        pos += 4
        end = pos + d * dt.itemsize
        if end > n:
            raise RuntimeError("I/O error: failed to fill whole buffer")
        out.append(buf[pos:end].view(dt))
        pos = end
    return out


def read_fvecs(path):
    """fvecs reader (src/formats.rs:7-47): a list of float lists."""
    return [v.tolist() for v in _read_vecs(path, "<f4")]


def read_ivecs(path):
    """ivecs reader (src/formats.rs:50-90): a list of int lists."""
    return [v.tolist() for v in _read_vecs(path, "<i4")]


def read_bvecs_as_f32(path):
    """bvecs reader with each byte scaled to [0, 1] as b / 255 in f32
    (src/formats.rs:93-122)."""
    return [(v.astype(np.float32) / np.float32(255.0)).tolist() for v in _read_vecs(path, np.uint8)]


def simd_info():
    """The reference reports which CPU SIMD sets its distance kernels use
    (src/metric.rs:41-60).  Here distances run in CUDA kernels for sm_100a
    (tensor-core MMAs for int8 and FP8), so this names that path."""
    return f"CUDA sm_100a kernels, libdgann ABI {_lib.lib().dg_version()}"


def write_fvecs(path, vectors):
    X = _f32(vectors)
    out = np.empty((X.shape[0], X.shape[1] + 1), dtype=np.int32)
    out[:, 0] = X.shape[1]
    out[:, 1:] = X.view(np.int32)
    out.tofile(path)


from .spfresh import SPFresh  # noqa: E402  (uses the helpers above)
from .incremental import IncrementalDiskANN  # noqa: E402
from .serve import Server, poisson_arrivals  # noqa: E402
