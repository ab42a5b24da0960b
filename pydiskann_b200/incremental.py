"""IncrementalDiskANN (diskann-rs src/incremental.rs): a base graph, a delta
layer of inserted vectors and tombstones, searched on the GPU as one graph.

The device index holds the reference's unified view (UnifiedView,
src/incremental.rs:349-471): base rows 0..base_count-1, then the delta rows,
then spare rows that nothing links to until a delta row is written there.
Inserts run DeltaLayer::add_vectors on the host (dg_delta_insert in
libdgann) and publish the new rows and the delta adjacency; deletes set bits
of a device tombstone bitmap.  Every search -- plain, filtered, batched --
is one dg_search_batch launch seeded with the base medoid and the delta
entry point.  Ids are the reference's: base ids as they are, delta ids
2^48 + local index (:334).
"""
from __future__ import annotations

import ctypes as C
import threading
import warnings

import numpy as np

from . import _lib
from . import formats as _fmt
from ._lib import PAD, check, lib, locked, ptr

DELTA_ID_OFFSET = 1 << 48
_METRICS = {"l2": _lib.L2SQ, "cosine": _lib.COSINE, "dot": _lib.DOT, "euclidean": _lib.L2}


class IncrementalDiskANN:
    """IncrementalDiskANN<D> with the binding's methods (python/src/lib.rs:126-205)."""

    def __init__(self, vectors, adjacency, medoid_id, metric="l2", labels=None, delta_threshold=10_000,
                 tombstone_ratio=0.1, delta_max_degree=32, device=0, quantizer=None, qparams=None, rerank_size=0,
                 base_codes=None):
        if metric not in _METRICS:
            raise ValueError(f"unknown metric: {metric}")
        X = np.ascontiguousarray(vectors, dtype=np.float32)
        A = np.ascontiguousarray(adjacency, dtype=np.uint32)
        if X.ndim != 2 or X.shape[0] == 0:
            raise RuntimeError("Index error: No vectors provided")
        self.metric_name, self.metric, self.device = metric, _METRICS[metric], device
        self.delta_threshold, self.tombstone_ratio = delta_threshold, tombstone_ratio
        self._bX, self._bA, self._bmed = X, A, int(medoid_id)
        self.dim = X.shape[1]
        self._dR = delta_max_degree  # IncrementalConfig::delta_params.max_degree (:31-43)
        self._dX = np.zeros((0, self.dim), np.float32)
        self._dA = np.zeros((0, self._dR), np.uint32)
        self._dn = 0
        self._ep = -1
        self._nf = 0 if labels is None else np.asarray(labels).shape[1]
        self._bL = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint64).reshape(len(X), -1)
        if self._bL is not None and len(self._bL) != len(X):
            raise RuntimeError(f"Index error: vectors.len() ({len(X)}) != labels.len() ({len(self._bL)})")
        self._dL = np.zeros((0, self._nf), np.uint64)
        self.tombstones: set[int] = set()
        # quantized base (build_quantized_*, src/incremental.rs:674-827): base rows
        # are scored by their codes, delta rows exactly; rerank_size reranks
        if quantizer not in (None, "f16", "int8", "pq", "rabitq"):
            raise ValueError(f"unknown quantizer: {quantizer}")
        self.quantizer, self._qp, self.rerank_size = quantizer, dict(qparams or {}), rerank_size
        self._base_codes = None if base_codes is None else np.ascontiguousarray(base_codes, dtype=np.uint8)
        self._ix = None
        self._cap = 0
        self._lock = threading.RLock()
        self._mirror(1024)

    # ------------------------------------------------------------ building
    @staticmethod
    def build(vectors, path=None, metric="l2", labels=None, quantizer=None, rerank_size=0, pq_subspaces=8,
              delta_threshold=10_000, tombstone_ratio=0.1, max_degree=64, build_beam_width=128, alpha=1.2,
              seed=0, device=0):
        """build_with_config / build_with_labels (src/incremental.rs:563-672): a
        Vamana base (GPU build) and an empty delta layer; writes the base core
        file at `path` when one is given."""
        import pydiskann_b200 as dg

        if quantizer not in (None, "f16", "int8", "pq", "rabitq"):
            raise ValueError(f"unknown quantizer: {quantizer}")
        X = np.ascontiguousarray(vectors, dtype=np.float32)
        if X.ndim != 2 or X.shape[0] == 0:
            raise RuntimeError("Index error: No vectors provided")
        if metric not in _METRICS:
            raise ValueError(f"unknown metric: {metric}")
        adj, med = dg.build_graph(X, max_degree, build_beam_width, alpha, metric, seed, None, device)
        if path is not None:
            _fmt.write_core(path, X, adj, med, metric)
        qp = {}
        if quantizer == "int8":  # trained on the build vectors, as build_quantized_int8
            qp["scale"], qp["offset"] = dg.int8_params(X)
        elif quantizer == "pq":
            qp["codebooks"] = dg.pq_train(X, pq_subspaces, 256, 20, 50_000, seed, device)
        elif quantizer == "rabitq":
            qp["centroid"], qp["signs"] = dg.rabitq_params(X, seed)
        return IncrementalDiskANN(X, adj, med, metric, labels, delta_threshold, tombstone_ratio, device=device,
                                  quantizer=quantizer, qparams=qp, rerank_size=rerank_size)

    @staticmethod
    def open(path, metric="l2", device=0):
        """open_with_config (src/incremental.rs:595-620): a DANN core file as the base."""
        if metric not in _METRICS:
            raise ValueError(f"unknown metric: {metric}")
        m, X, A = _fmt.read_core(path)
        if m.distance_name != _fmt.DISTANCE_NAMES[metric]:
            warnings.warn(f"index recorded distance `{m.distance_name}` but you opened with "
                          f"`{_fmt.DISTANCE_NAMES[metric]}`", RuntimeWarning, stacklevel=2)
        return IncrementalDiskANN(X, A, m.medoid_id, metric, device=device)

    # ------------------------------------------------------------ device mirror
    @property
    def base_count(self):
        return len(self._bX)

    def _delta_rows(self, j0, j1):
        """Unified vectors / adjacency / labels of delta rows [j0, j1): local
        neighbour ids shifted by base_count (UnifiedView::get_neighbors, :430-450)."""
        nb = self.base_count
        dA = self._dA[j0:j1]
        A = np.full((j1 - j0, self._Ru), PAD, np.uint32)
        A[:, : dA.shape[1]] = np.where(dA != PAD, dA + np.uint32(nb), np.uint32(PAD))
        L = np.ascontiguousarray(self._dL[j0:j1]) if self._nf else None
        return np.ascontiguousarray(self._dX[j0:j1]), A, L

    def _mirror(self, delta_cap):
        """(Re)creates the device index with room for delta_cap delta rows."""
        self.close()
        nb = self.base_count
        self._Ru = max(self._bA.shape[1], self._dR)
        self._cap = delta_cap
        n = nb + delta_cap
        X = np.zeros((n, self.dim), np.float32)
        X[:nb] = self._bX
        X[nb: nb + self._dn] = self._dX[: self._dn]
        A = np.full((n, self._Ru), PAD, np.uint32)
        A[:nb, : self._bA.shape[1]] = self._bA
        if self._dn:
            A[nb: nb + self._dn] = self._delta_rows(0, self._dn)[1]
        import pydiskann_b200 as dg

        if self.quantizer is None:
            self._ix = dg._Index(X, A, self._bmed, self.metric_name, self.device)
        else:
            self._ix = dg.QuantizedDiskANN(X, A, self._bmed, self.metric_name, self.device, self.rerank_size)
            self._attach_codes(n)
        self._h = self._ix._h
        if self._nf:
            Lb = np.zeros((n, self._nf), np.uint64)
            Lb[:nb] = self._bL
            Lb[nb: nb + self._dn] = self._dL[: self._dn]
            check(lib().dg_index_attach_labels(self._h, self._nf, ptr(Lb)))
        if getattr(self, "_bf16", False):
            self._ix.enable_bf16()
        self._publish_seeds()
        self._publish_tombstones(list(self.tombstones))

    def _attach_codes(self, n):
        """Codes of the base rows (given, or encoded on the GPU); rows past the
        base carry none (dg_index_set_code_limit)."""
        codes = None
        if self._base_codes is not None:
            codes = np.zeros((n, self._base_codes.shape[1]), np.uint8)
            codes[: self.base_count] = self._base_codes
        q, p = self.quantizer, self._qp
        if q == "int8":
            self._ix.attach_int8(p["scale"], p["offset"], codes)
        elif q == "f16":
            self._ix.attach_f16(None if codes is None else codes.view(np.uint16))
        elif q == "pq":
            self._ix.attach_pq(p["codebooks"], codes)
        else:
            self._ix.attach_rabitq(p["centroid"], p["signs"], codes)
        check(lib().dg_index_set_code_limit(self._ix._h, self.base_count))

    def _publish_seeds(self):
        """UnifiedView::entry_points (src/incremental.rs:383-392)."""
        seeds = [self._bmed] + ([self.base_count + self._ep] if self._ep >= 0 else [])
        arr = np.asarray(seeds, np.uint32)
        check(lib().dg_index_set_entry_points(self._h, ptr(arr), len(arr)))

    def _row_of(self, gid):
        gid = int(gid)
        if gid >= DELTA_ID_OFFSET:
            j = gid - DELTA_ID_OFFSET
            return self.base_count + j if j < self._dn else None
        return gid if gid < self.base_count else None

    def _publish_tombstones(self, gids, deleted=1):
        rows = [r for r in (self._row_of(g) for g in gids) if r is not None]
        arr = np.asarray(rows if rows else [0], np.uint32)
        check(lib().dg_index_set_tombstones(self._h, ptr(arr), len(rows), deleted, len(self.tombstones)))

    @locked
    def close(self):
        if getattr(self, "_ix", None) is not None:
            self._ix.close()
            self._ix = None
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ updates
    def add_vectors(self, vectors):
        """add_vectors (src/incremental.rs:829-857): new ids 2^48 + local index."""
        if len(vectors) == 0:
            return []
        X = _lib.rows_f32(vectors, self.dim, self._dim_error)
        return self._add(X, None)

    def _dim_error(self, i, n):
        return f"Index error: Vector {i} has dimension {n} but index expects {self.dim}"

    def add_vectors_with_labels(self, vectors, labels):
        """add_vectors_with_labels (src/incremental.rs:859-906)."""
        if len(vectors) == 0:
            return []
        lab = [list(map(int, l)) for l in labels]
        if len(lab) != len(vectors):
            raise RuntimeError(f"Index error: vectors.len() ({len(vectors)}) != labels.len() ({len(lab)})")
        X = _lib.rows_f32(vectors, self.dim, self._dim_error)
        for i, l in enumerate(lab):
            if self._nf > 0 and len(l) != self._nf:
                raise RuntimeError(f"Index error: Label {i} has {len(l)} fields, expected {self._nf}")
        return self._add(X, np.asarray(lab, dtype=np.uint64).reshape(len(X), self._nf))

    @locked
    def _add(self, X, labels):
        n_old, n_new = self._dn, len(X)
        need = n_old + n_new
        if need > len(self._dX):
            grow = max(need, 2 * len(self._dX), 1024)
            dX = np.zeros((grow, self.dim), np.float32)
            dX[:n_old] = self._dX[:n_old]
            dA = np.full((grow, self._dR), PAD, np.uint32)
            dA[:n_old] = self._dA[:n_old]
            dL = np.zeros((grow, self._nf), np.uint64)
            dL[:n_old] = self._dL[:n_old]
            self._dX, self._dA, self._dL = dX, dA, dL
        self._dX[n_old:need] = X
        if self._nf:
            self._dL[n_old:need] = 0 if labels is None else labels
        ep = C.c_int64(self._ep)
        check(lib().dg_delta_insert(ptr(self._dX), self.dim, self.metric, self._dR, ptr(self._dA), n_old, n_new,
                                    C.byref(ep)))
        self._dn, self._ep = need, ep.value
        if need > self._cap:
            self._mirror(max(need, 2 * self._cap, 1024))
        else:
            nb = self.base_count
            # new rows, then every delta adjacency row (back-edges rewrote old ones)
            Xn, _, Ln = self._delta_rows(n_old, need)
            check(lib().dg_index_update_rows(self._h, nb + n_old, n_new, ptr(Xn), None, ptr(Ln)))
            Ad = self._delta_rows(0, need)[1]
            check(lib().dg_index_update_rows(self._h, nb, need, None, ptr(Ad), None))
            self._publish_seeds()
            born = [g for g in range(DELTA_ID_OFFSET + n_old, DELTA_ID_OFFSET + need) if g in self.tombstones]
            if born:  # ids deleted before they were inserted
                self._publish_tombstones(born)
        return [DELTA_ID_OFFSET + j for j in range(n_old, need)]

    @locked
    def delete_vectors(self, ids):
        """delete_vectors (src/incremental.rs:908-915): tombstones."""
        new = [int(i) for i in ids if int(i) not in self.tombstones]
        self.tombstones.update(new)
        self._publish_tombstones(new)

    @locked
    def is_deleted(self, id):  # noqa: A002
        return int(id) in self.tombstones

    # ------------------------------------------------------------ search
    def _to_global(self, ids, cnt):
        nb = self.base_count
        g = ids.astype(np.uint64)
        delta = (ids != PAD) & (ids >= nb)
        g[delta] = np.uint64(DELTA_ID_OFFSET) + (ids[delta].astype(np.uint64) - np.uint64(nb))
        return g

    @locked
    def search_arrays(self, queries, k=10, beam_width=128, filters=None, traversal=None, rerank_size=None):
        """Batched search: (ids u64[nq, k], dists f32[nq, k], counts u32[nq]).
        A filter only applies to an index with labels, as in
        search_filtered_with_dists (src/incremental.rs:1020-1030)."""
        Q = _lib.query_rows(queries, self.dim)
        if filters is not None and not self._nf:
            filters = None
        if traversal is None:  # the quantizer's codes unless a label filter is given (:1020-1070)
            traversal = _lib.TRAVERSE_CODES if self.quantizer and filters is None else _lib.TRAVERSE_F32
        if rerank_size is None:
            rerank_size = self.rerank_size if traversal == _lib.TRAVERSE_CODES else 0
        ids, ds, cnt = _mirror_search(self._ix, Q, k, beam_width, traversal, rerank_size, filters)
        return self._to_global(ids, cnt), ds, cnt

    @locked
    def enable_bf16(self):
        """BF16 copy of the unified rows for ``traversal=TRAVERSE_BF16`` (kept in
        step with inserts); no counterpart in the reference."""
        self._ix.enable_bf16()
        self._bf16 = True

    def search_with_dists(self, query, k=10, beam_width=128):
        ids, ds, cnt = self.search_arrays(np.asarray(query, np.float32).reshape(1, -1), k, beam_width)
        return [(int(ids[0, j]), float(ds[0, j])) for j in range(int(cnt[0]))]

    def search(self, query, k=10, beam_width=128):
        return [i for i, _ in self.search_with_dists(query, k, beam_width)]

    def search_filtered_with_dists(self, query, filter, k=10, beam_width=128):  # noqa: A002
        ids, ds, cnt = self.search_arrays(np.asarray(query, np.float32).reshape(1, -1), k, beam_width, filter)
        return [(int(ids[0, j]), float(ds[0, j])) for j in range(int(cnt[0]))]

    def search_filtered(self, query, filter, k=10, beam_width=128):  # noqa: A002
        return [i for i, _ in self.search_filtered_with_dists(query, filter, k, beam_width)]

    def search_batch(self, queries, k=10, beam_width=128):
        ids, _, cnt = self.search_arrays(queries, k, beam_width)
        return [ids[i, : cnt[i]].astype(np.int64).tolist() for i in range(len(cnt))]

    # ------------------------------------------------------------ state
    @locked
    def get_vector(self, id):  # noqa: A002
        """get_vector (src/incremental.rs:1083-1098)."""
        id = int(id)  # noqa: A001
        if id >= DELTA_ID_OFFSET:
            j = id - DELTA_ID_OFFSET
            return self._dX[j].tolist() if j < self._dn else None
        return self._bX[id].tolist() if id < self.base_count else None

    @locked
    def should_compact(self):
        """should_compact (src/incremental.rs:1100-1122)."""
        if self._dn >= self.delta_threshold:
            return True
        total = self.base_count + self._dn
        return total > 0 and np.float32(len(self.tombstones)) / np.float32(total) >= np.float32(self.tombstone_ratio)

    @locked
    def compact(self, new_path=None, max_degree=None, build_beam_width=128, alpha=1.2, seed=0):
        """compact (src/incremental.rs:1124-1205): the live base and delta rows, in
        id order, become a new base (Vamana graph built on the GPU); the delta
        layer and the tombstones are cleared.  Base ids are renumbered."""
        import pydiskann_b200 as dg

        live_b = [i for i in range(self.base_count) if i not in self.tombstones]
        live_d = [j for j in range(self._dn) if DELTA_ID_OFFSET + j not in self.tombstones]
        if not live_b and not live_d:
            raise RuntimeError("Index error: Cannot compact: no vectors remaining after removing tombstones")
        X = np.concatenate([self._bX[live_b], self._dX[live_d]]).astype(np.float32)
        L = None
        if self._nf:
            L = np.concatenate([self._bL[live_b], self._dL[live_d]])
        R = max_degree or self._bA.shape[1]
        adj, med = dg.build_graph(X, R, build_beam_width, alpha, self.metric_name, seed, None, self.device)
        if new_path is not None:
            _fmt.write_core(new_path, X, adj, med, self.metric_name)
        self._bX, self._bA, self._bmed, self._bL = X, adj, int(med), L
        self._base_codes = None  # re-encoded with the same quantizer (:1180-1190)
        self._dX = np.zeros((0, self.dim), np.float32)
        self._dA = np.zeros((0, self._dR), np.uint32)
        self._dL = np.zeros((0, self._nf), np.uint64)
        self._dn, self._ep = 0, -1
        self.tombstones = set()
        self._mirror(1024)

    @locked
    def stats(self):
        """stats (src/incremental.rs:1613-1626)."""
        nb = self.base_count
        return {"base_vectors": nb, "delta_vectors": self._dn, "tombstones": len(self.tombstones),
                "total_live": max(nb + self._dn - len(self.tombstones), 0), "dim": self.dim}

    # ------------------------------------------------------------ persistence
    @locked
    def to_bytes(self) -> bytes:
        """IncrementalDiskANN::to_bytes (src/incremental.rs:1234-1327)."""
        graph = [row[row != PAD].tolist() for row in self._dA[: self._dn]]
        labels = None
        if self._nf:
            labels = (self._nf, self._bL, self._dL[: self._dn])
        base = _fmt.core_bytes(self._bX, self._bA, self._bmed, self.metric_name)
        quant = None
        if self.quantizer:
            st = self._state()
            quant = (st.code_size, self.rerank_size, st, self._ix.codes()[: self.base_count])
        return _fmt.incremental_bytes(self._dX[: self._dn], graph, None if self._ep < 0 else self._ep, self._dR,
                                      sorted(self.tombstones), base=base, labels=labels, dim=self.dim,
                                      quantizer=quant)

    def _state(self):
        """The quantizer as the serialized QuantizerState."""
        q, p = self.quantizer, self._qp
        if q == "int8":
            return _fmt.QuantizerState("int8", self.dim, scale=float(p["scale"]), offset=float(p["offset"]))
        if q == "f16":
            return _fmt.QuantizerState("f16", self.dim)
        if q == "pq":
            cb = np.asarray(p["codebooks"], np.float32)
            return _fmt.QuantizerState("pq", self.dim, *cb.shape, codebooks=cb.reshape(-1))
        sg = np.asarray(p["signs"], np.float32)
        return _fmt.QuantizerState("rabitq", self.dim, padded=sg.size // 3,
                                   centroid=np.asarray(p["centroid"], np.float32), signs=sg)

    @staticmethod
    def from_bytes(data, metric="l2", device=0):
        """IncrementalDiskANN::from_bytes (src/incremental.rs:1332-1611), INCR v2."""
        if metric not in _METRICS:
            raise ValueError(f"unknown metric: {metric}")
        p = _fmt.parse_incremental(data)
        if p["base"] is None:
            raise RuntimeError("Index error: an incremental index without a base layer is not supported")
        m, X, A = _fmt.parse_core(p["base"])
        lab = p["labels"]
        qz = p["quantizer"]
        kw = {}
        if qz is not None:
            code_size, rerank, st, codes = qz
            if st.dim != m.dim or codes.size != m.num_vectors * code_size:
                raise RuntimeError("Index error: quantizer section does not match the base index")
            qp = {"int8": lambda: {"scale": st.scale, "offset": st.offset}, "f16": lambda: {},
                  "pq": lambda: {"codebooks": st.codebooks.reshape(st.num_subspaces, st.num_centroids,
                                                                   st.subspace_dim)},
                  "rabitq": lambda: {"centroid": st.centroid, "signs": st.signs}}[st.kind]()
            kw = {"quantizer": st.kind, "qparams": qp, "rerank_size": int(rerank),
                  "base_codes": codes.reshape(m.num_vectors, code_size)}
        ix = IncrementalDiskANN(X, A, m.medoid_id, metric, None if lab is None else lab[1], device=device, **kw)
        ix._dR = max(int(p["max_degree"]), max((len(g) for g in p["graph"]), default=0), 1)
        dn = len(p["vectors"])
        ix._dX = np.array(p["vectors"], dtype=np.float32).reshape(dn, ix.dim)
        ix._dA = np.full((dn, ix._dR), PAD, np.uint32)
        for j, g in enumerate(p["graph"]):
            if any(x >= dn for x in g):
                raise RuntimeError("Index error: delta graph id out of range")
            ix._dA[j, : len(g)] = g
        ix._dL = np.zeros((dn, ix._nf), np.uint64) if lab is None else np.asarray(lab[2], np.uint64).reshape(dn, -1)
        ix._dn = dn
        ix._ep = -1 if p["entry_point"] is None else int(p["entry_point"])
        if ix._ep >= dn:
            raise RuntimeError("Index error: delta entry point out of range")
        ix.tombstones = set(int(t) for t in p["tombstones"])
        ix._mirror(max(1024, dn))
        return ix


def _mirror_search(ix, Q, k, L, traversal, rerank_size, filters):
    """The mirror's batched search with the base class's argument order (a
    QuantizedDiskANN mirror defaults its traversal and rerank otherwise)."""
    import pydiskann_b200 as dg

    return dg._Index.search_arrays(ix, Q, k, L, traversal, rerank_size, filters=filters)
