"""SPFresh (diskann-rs src/spfresh.rs): posting lists searched on the GPU,
maintained on the host.

Search runs in libdgann (dg_spfresh_search_batch): routing to the nprobe
nearest live postings, the probe_ratio cut, the scan with tombstones and the
FP32 rerank, or the RaBitQ error-bound scan.  This module holds the host side
of the index the way the reference keeps it -- posting slots with
(id, code) entries, centroids, a raw vector store, tombstones -- and restates
its update path: insert (nearest posting, push, split when full,
src/spfresh.rs:416-476), drain / split with 2-means and neighbourhood
reassignment (:122-162, 502-611), relocate (:538-573) and gc (:613-643).
Routing is brute force over the live centroids at every size (the reference
switches to a centroid graph above 4096 postings, :358-378; that graph is
rebuilt non-deterministically, so exact routing is used instead).  Changed
posting slots are uploaded to the device after each call.
"""
from __future__ import annotations

import ctypes as C
import math
import threading

import numpy as np

from . import _lib
from ._lib import check, lib, locked, ptr

_METRICS = {"l2": _lib.L2SQ, "cosine": _lib.COSINE, "dot": _lib.DOT, "euclidean": _lib.L2}
CHUNK = 4096


def _seq_rows(metric, v, C_):
    """metric_eval(v, c) for every row c of C_, summed in coordinate order in
    f32: the arithmetic of the GPU routing kernels (seq_metric) and of the
    oracle's metric_eval, i.e. the reference's f32 distances in a fixed order."""
    Ct = np.ascontiguousarray(np.asarray(C_, dtype=np.float32).T)
    v = np.asarray(v, dtype=np.float32).reshape(-1)
    n = Ct.shape[1]
    if metric in (_lib.L2SQ, _lib.L2):
        acc = np.zeros(n, dtype=np.float32)
        for i in range(len(v)):
            t = v[i] - Ct[i]
            acc = acc + t * t
        return np.sqrt(acc) if metric == _lib.L2 else acc
    ab = np.zeros(n, dtype=np.float32)
    bb = np.zeros(n, dtype=np.float32)
    aa = np.float32(0.0)
    for i in range(len(v)):
        ab = ab + v[i] * Ct[i]
        aa = np.float32(aa + v[i] * v[i])
        bb = bb + Ct[i] * Ct[i]
    if metric == _lib.DOT:
        return np.float32(1.0) - ab
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.float32(1.0) - ab / (np.sqrt(aa) * np.sqrt(bb))
    r = np.where((aa == 0) & (bb == 0), np.float32(0.0), np.where(ab == 0, np.float32(1.0), r))
    return np.maximum(r, np.float32(0.0)).astype(np.float32)


def _seq_matrix(metric, V, C_):
    """_seq_rows for every row of V: an f32 [len(V), len(C_)] matrix."""
    V = np.asarray(V, dtype=np.float32)
    C_ = np.asarray(C_, dtype=np.float32)
    out = np.empty((len(V), len(C_)), dtype=np.float32)
    if len(V) == 0 or len(C_) == 0:
        return out
    if metric in (_lib.L2SQ, _lib.L2):
        acc = np.zeros((len(V), len(C_)), dtype=np.float32)
        for i in range(V.shape[1]):
            t = V[:, i, None] - C_[None, :, i]
            acc = acc + t * t
        return np.sqrt(acc) if metric == _lib.L2 else acc
    for r in range(len(V)):
        out[r] = _seq_rows(metric, V[r], C_)
    return out


def _fht(v):
    """Unnormalised fast Walsh-Hadamard transform along the last axis (src/rabitq.rs:31-43)."""
    v = v.copy()
    n = v.shape[-1]
    h = 1
    while h < n:
        a = v.reshape(*v.shape[:-1], n // (2 * h), 2, h)
        x, y = a[..., 0, :].copy(), a[..., 1, :].copy()
        a[..., 0, :] = x + y
        a[..., 1, :] = x - y
        h *= 2
    return v


class _Codec:
    """Code of a vector stored in a posting (Inner::encode, src/spfresh.rs:328-339)."""

    def __init__(self, kind, dim, params, device=None):
        self.kind, self.dim, self.p = kind, dim, params
        self.device = device  # RaBitQ residual codes are encoded on this GPU (None: on the host)
        if kind is None:
            self.size = 4 * dim
        elif kind == "f16":
            self.size = 2 * dim
        elif kind == "int8":
            self.size = dim
        elif kind == "pq":
            self.size = params["codebooks"].shape[0]
        else:
            self.size = params["padded"] // 8 + 8

    @property
    def residual(self):
        return self.kind == "rabitq"

    def encode(self, V, centroid=None):
        V = np.atleast_2d(np.asarray(V, dtype=np.float32))
        if self.kind is None:
            return V.view(np.uint8).reshape(len(V), -1).copy()
        if self.kind == "f16":
            return V.astype(np.float16).view(np.uint8).reshape(len(V), -1).copy()
        if self.kind == "int8":
            s, o = np.float32(self.p["scale"]), np.float32(self.p["offset"])
            t = V * (np.float32(1.0) / s) + (-o / s)
            return np.clip(np.rint(t), 0, 255).astype(np.uint8)
        if self.kind == "pq":
            cb = self.p["codebooks"]
            M, K, ds = cb.shape
            out = np.empty((len(V), M), dtype=np.uint8)
            for m in range(M):
                sub = V[:, m * ds:(m + 1) * ds]
                d = ((sub[:, None, :] - cb[m][None]) ** 2).sum(-1, dtype=np.float32)
                out[:, m] = d.argmin(1)
            return out
        # RaBitQ residual code against the posting centroid (src/rabitq.rs:218-256)
        if self.device is not None:
            import pydiskann_b200 as dg

            return dg.rabitq_encode(V, centroid, self.p["signs"], self.p["padded"], self.device)
        P, signs = self.p["padded"], self.p["signs"].reshape(3, -1)
        r = np.zeros((len(V), P), dtype=np.float32)
        r[:, : self.dim] = V - centroid
        norm = np.sqrt((r * r).sum(1, dtype=np.float32)).astype(np.float32)
        nz = norm > 0
        r[nz] /= norm[nz, None]
        for rd in range(3):
            r = _fht(r * signs[rd])
        bits = np.packbits(r > 0, axis=1, bitorder="little")
        ip = np.abs(r).sum(1, dtype=np.float32) / np.float32(math.sqrt(P))
        fac = np.where(ip > 0, norm / np.where(ip > 0, ip, 1), 0).astype(np.float32)
        tail = np.stack([norm * norm, fac], 1).astype(np.float32).view(np.uint8)
        return np.concatenate([bits, tail], 1)


def kmeans2(vs, metric):
    """2-means on raw vectors with an index split when degenerate (src/spfresh.rs:122-162)."""
    n = len(vs)

    def means(side):
        out = []
        for k in (False, True):
            sel = vs[side == k]
            cnt = max(len(sel), 1)
            out.append((sel.sum(0, dtype=np.float32) / np.float32(cnt)).astype(np.float32))
        return out

    d0 = _seq_rows(metric, vs[0], vs[1:]) if n > 1 else np.zeros(0)
    far = int(np.argmax(d0)) + 1 if n > 1 else 0
    c = [vs[0].copy(), vs[far].copy()]
    side = np.zeros(n, dtype=bool)
    for _ in range(5):
        side = _seq_rows(metric, c[1], vs) < _seq_rows(metric, c[0], vs)
        if side.all() or not side.any():
            break
        c = means(side)
    if side.all() or not side.any():
        side = np.arange(n) >= n // 2
        c = means(side)
    return c[0], c[1], side


class SPFresh:
    """SPFresh<D> (src/spfresh.rs:774-936) with GPU posting scans."""

    def __init__(self, dim, metric="l2", quantizer=None, qparams=None, rerank_size=0, max_posting_size=128,
                 min_posting_size=16, reassign_neighbors=16, probe_ratio=float("inf"), device=0):
        if metric not in _METRICS:
            raise ValueError(f"unknown metric: {metric}")
        self.dim, self.metric_name, self.metric = dim, metric, _METRICS[metric]
        self.codec = _Codec(quantizer, dim, qparams or {}, device)
        self.rerank_size, self.max_posting, self.min_posting = rerank_size, max_posting_size, min_posting_size
        self.reassign_neighbors, self.probe_ratio, self.device = reassign_neighbors, probe_ratio, device
        self.cap = 2 * max_posting_size  # block layout, src/spfresh.rs:109-111
        self.cent = np.zeros((0, dim), dtype=np.float32)
        self.live_b = np.zeros(0, dtype=bool)
        self.ids = []      # per slot: np.uint64 array of entry ids
        self.codes = []    # per slot: u8 [len, code_size]
        # freed slots with the epoch that freed them; a slot is reused only in
        # a later epoch (an insert chunk or a gc), src/spfresh.rs:380-415
        self.free = []
        self.epoch = 1
        self.raw = np.zeros((0, dim), dtype=np.float32)
        self.next_id = 0
        self.deleted = set()
        self.live = 0
        self.created = []
        self._h = None
        self._dirty = set()
        self._cent_dirty = set()  # slots whose centroid or live flag the device mirror has not seen
        self._dev_blocks = 0
        self._dev_ids = 0
        self._raw_synced = 0
        self._del_synced = set()
        self.centroid_beam = 64  # SPFreshConfig::centroid_beam, kept for the saved config
        self.path = None
        self._lock = threading.RLock()

    # ------------------------------------------------------------ building
    @staticmethod
    def build(vectors, path=None, metric="l2", quantizer=None, rerank_size=0, pq_subspaces=8,
              max_posting_size=128, min_posting_size=16, reassign_neighbors=16, probe_ratio=float("inf"),
              seed=0, device=0):
        """SPFresh::build (src/spfresh.rs:801-817): n / (max_posting/2) postings seeded
        from random vectors, then every vector inserted."""
        X = np.ascontiguousarray(vectors, dtype=np.float32)
        if X.ndim != 2 or len(X) == 0:
            raise RuntimeError("Index error: No vectors provided")
        if quantizer not in (None, "f16", "int8", "pq", "rabitq"):
            raise ValueError(f"unknown quantizer: {quantizer}")
        import pydiskann_b200 as dg

        qp = {}
        if quantizer == "pq" and device is None:
            raise ValueError("PQ training runs on the GPU; give a device")
        if quantizer == "int8":
            qp["scale"], qp["offset"] = dg.int8_params(X)
        elif quantizer == "pq":
            qp["codebooks"] = dg.pq_train(X, pq_subspaces, 256, 20, 50_000, seed, device)
        elif quantizer == "rabitq":
            cen, signs = dg.rabitq_params(X, seed)
            qp["padded"], qp["signs"], qp["centroid"] = dg.rabitq_padded(X.shape[1]), signs, cen
        s = SPFresh(X.shape[1], metric, quantizer, qp, rerank_size, max_posting_size, min_posting_size,
                    reassign_neighbors, probe_ratio, device)
        k = max(1, len(X) // max(max_posting_size // 2, 1))
        rng = np.random.default_rng([seed, 0x5EED])
        for i in rng.choice(len(X), size=min(k, len(X)), replace=False):
            s._new_posting(X[i].copy())
        s._insert(X)
        s._sync()
        if path is not None:  # SPFresh::build saves at `path` (src/spfresh.rs:785-817)
            s.save(path)
        return s

    @staticmethod
    def bulk_load(vectors, metric="l2", quantizer=None, qparams=None, rerank_size=0, max_posting_size=128,
                  min_posting_size=16, reassign_neighbors=16, probe_ratio=float("inf"), seed=0, device=0):
        """Postings from a nearest-centroid assignment instead of one insert per
        vector: n / (max_posting / 2) centroids sampled from the vectors (as
        SPFresh::build seeds them, src/spfresh.rs:801-807), every vector assigned
        to its nearest centroid on the GPU (exact), and postings above
        max_posting_size split by the same 2-means as an insert-time split
        (without relocating neighbours).  The result satisfies the index's
        invariants, so inserts, deletes and searches continue as after build();
        it is for large loads, where per-vector insertion is host-bound.
        Quantizer parameters default as in build() (int8 range, PQ with 8
        subspaces, RaBitQ rotation signs and centroid)."""
        import pydiskann_b200 as dg

        X = np.ascontiguousarray(vectors, dtype=np.float32)
        if X.ndim != 2 or len(X) == 0:
            raise RuntimeError("Index error: No vectors provided")
        if device is None:
            raise ValueError("bulk_load assigns on the GPU; give a device")
        qp = dict(qparams or {})
        if quantizer == "int8" and not qp:
            qp["scale"], qp["offset"] = dg.int8_params(X)
        elif quantizer == "pq" and not qp:
            qp["codebooks"] = dg.pq_train(X, 8, 256, 20, 50_000, seed, device)
        elif quantizer == "rabitq" and not qp:
            cen, signs = dg.rabitq_params(X, seed)
            qp["padded"], qp["signs"], qp["centroid"] = dg.rabitq_padded(X.shape[1]), signs, cen
        s = SPFresh(X.shape[1], metric, quantizer, qp, rerank_size, max_posting_size, min_posting_size,
                    reassign_neighbors, probe_ratio, device)
        n = len(X)
        k = max(1, n // max(max_posting_size // 2, 1))
        rng = np.random.default_rng([seed, 0x5EED])
        C = X[rng.choice(n, size=min(k, n), replace=False)]
        assign, _ = dg.exact_knn(C, X, 1, metric=metric, device=device)
        assign = assign[:, 0].astype(np.int64)
        order = np.argsort(assign, kind="stable")
        bounds = np.searchsorted(assign[order], np.arange(len(C) + 1))
        queue = [(C[c], order[bounds[c]:bounds[c + 1]]) for c in range(len(C)) if bounds[c + 1] > bounds[c]]
        finals = []
        while queue:
            c, mem = queue.pop()
            if len(mem) > max_posting_size:
                c1, c2, side = kmeans2(X[mem], s.metric)
                queue.append((c1, mem[~side]))
                queue.append((c2, mem[side]))
            else:
                finals.append((np.asarray(c, dtype=np.float32), mem))
        s.cent = np.stack([c for c, _ in finals]).astype(np.float32)
        s.live_b = np.ones(len(finals), dtype=bool)
        s.ids = [mem.astype(np.uint64) for _, mem in finals]
        s.codes = [s.codec.encode(X[mem], s.cent[b] if s.codec.residual else None) for b, (_, mem) in enumerate(finals)]
        s._dirty = set(range(len(finals)))
        s.raw = X.copy()
        s.next_id = n
        s.live = n
        s._sync()
        return s

    # ------------------------------------------------------------ host state
    def _len(self, b):
        return len(self.ids[b])

    def _is_live(self, b):
        return 0 <= b < len(self.live_b) and bool(self.live_b[b])

    def _live_entries(self, b):
        ids, codes = self.ids[b], self.codes[b]
        keep = np.array([int(i) not in self.deleted for i in ids], dtype=bool) if len(ids) else np.zeros(0, bool)
        return ids[keep], codes[keep]

    def _alloc_free(self):
        """Inner::alloc (src/spfresh.rs:380-393): the first freed slot of an
        earlier epoch, taken out by swap-remove; None when there is none."""
        for i, (b, e) in enumerate(self.free):
            if e < self.epoch:
                self.free[i] = self.free[-1]
                self.free.pop()
                return b
        return None

    def _new_posting(self, centroid):
        b = self._alloc_free()
        if b is not None:
            self.cent[b] = centroid
        else:
            b = len(self.live_b)
            self.cent = np.vstack([self.cent, centroid[None].astype(np.float32)])
            self.live_b = np.append(self.live_b, False)
            self.ids.append(np.zeros(0, dtype=np.uint64))
            self.codes.append(np.zeros((0, self.codec.size), dtype=np.uint8))
        self.live_b[b] = True
        self.ids[b] = np.zeros(0, dtype=np.uint64)
        self.codes[b] = np.zeros((0, self.codec.size), dtype=np.uint8)
        self.created.append(b)
        self._dirty.add(b)
        self._cent_dirty.add(b)
        return b

    def _free_posting(self, b):
        self.live_b[b] = False
        self.ids[b] = np.zeros(0, dtype=np.uint64)
        self.codes[b] = np.zeros((0, self.codec.size), dtype=np.uint8)
        self.free.append((b, self.epoch))
        self._dirty.add(b)
        self._cent_dirty.add(b)

    def _rewrite(self, b, ids, codes):
        self.ids[b], self.codes[b] = np.asarray(ids, dtype=np.uint64), np.asarray(codes, dtype=np.uint8).reshape(-1, self.codec.size)
        self._dirty.add(b)

    def _push(self, b, id_, code):
        self.ids[b] = np.append(self.ids[b], np.uint64(id_))
        self.codes[b] = np.vstack([self.codes[b], np.asarray(code, dtype=np.uint8).reshape(1, -1)])
        self._dirty.add(b)

    def _encode(self, v, b):
        return self.codec.encode(v, self.cent[b] if self.codec.residual else None)[0]

    def _device_routing(self):
        """True when the device mirror can route against the current postings:
        it exists and holds every slot; new and freed postings are published
        first (their centroids and live flags)."""
        if self._h is None:
            return False
        if len(self.live_b) > self._dev_blocks:
            self._create_device()
            return True
        if self._cent_dirty:
            blocks = np.array(sorted(self._cent_dirty), dtype=np.uint32)
            cent = np.ascontiguousarray(self.cent[blocks], dtype=np.float32)
            live = np.ascontiguousarray(self.live_b[blocks], dtype=np.uint8)
            check(lib().dg_spfresh_set_centroids(self._h, ptr(blocks), len(blocks), ptr(cent), ptr(live)))
            self._cent_dirty.clear()
        return True

    def _nearest_many(self, V, n):
        """Inner::nearest (src/spfresh.rs:358-378) for every row of V: the n
        nearest live postings as (slots, distances), ascending by (distance,
        slot), FP32 coordinate-order distances; on the GPU when the device
        mirror is attached (dg_spfresh_nearest), else on the host."""
        V = np.ascontiguousarray(V, dtype=np.float32).reshape(-1, self.dim)
        live = np.nonzero(self.live_b)[0]
        n = min(n, len(live))
        if n == 0 or len(V) == 0:
            return np.zeros((len(V), 0), np.int64), np.zeros((len(V), 0), np.float32)
        if n <= 64 and self._device_routing():
            slots = np.empty((len(V), n), dtype=np.uint32)
            dists = np.empty((len(V), n), dtype=np.float32)
            check(lib().dg_spfresh_nearest(self._h, ptr(V), len(V), n, ptr(slots), ptr(dists)))
            return slots.astype(np.int64), dists
        D = _seq_matrix(self.metric, V, self.cent[live])
        order = np.lexsort((np.broadcast_to(live, D.shape), D), axis=1)[:, :n]
        return live[order], np.take_along_axis(D, order, axis=1)

    def _nearest(self, v, n):
        """Live postings by (distance to centroid, slot), closest first (src/spfresh.rs:358-378)."""
        slots, dists = self._nearest_many(v, n)
        return [(int(b), float(d)) for b, d in zip(slots[0], dists[0])]

    def _dist(self, v, b):
        return float(_seq_rows(self.metric, v, self.cent[b:b + 1])[0])

    # --------------------------------------------------------------- updates
    @locked
    def insert(self, vectors):
        """Inner::insert (src/spfresh.rs:416-476); returns the new ids."""
        X = _lib.rows_f32(vectors, self.dim, lambda i, n: f"Index error: Vector dim {n} != index dim {self.dim}")
        ids = self._insert(X)
        self._sync()
        return ids

    def _insert(self, X):
        first = self.next_id
        ids = list(range(first, first + len(X)))
        if first + len(X) > len(self.raw):
            grow = np.zeros((max(first + len(X), 2 * len(self.raw)) - len(self.raw), self.dim), dtype=np.float32)
            self.raw = np.vstack([self.raw, grow])
        self.raw[first:first + len(X)] = X
        self.next_id += len(X)
        self.live += len(X)
        for c0 in range(0, len(X), CHUNK):
            chunk = X[c0:c0 + CHUNK]
            self.epoch += 1
            self.created = []
            # nearest live posting per vector (lowest slot on ties), as the
            # reference routes a chunk before inserting it
            slots, _ = self._nearest_many(chunk, 1)
            targets = [int(t) for t in slots[:, 0]] if slots.shape[1] else [None] * len(chunk)
            for j, v in enumerate(chunk):
                id_ = first + c0 + j
                t = targets[j]
                best = (t, self._dist(v, t)) if t is not None and self._is_live(t) else None
                if best is None:
                    nn = self._nearest(v, 1)
                    best = nn[0] if nn else None
                cr = [c for c in self.created if self._is_live(c)]
                if cr:  # postings split off earlier in this chunk
                    dc = _seq_rows(self.metric, v, self.cent[cr])
                    for c, dd in zip(cr, dc):
                        if best is None or dd < best[1]:
                            best = (c, float(dd))
                b = best[0] if best is not None else self._new_posting(v.copy())
                self._push(b, id_, self._encode(v, b))
                if self._len(b) >= self.max_posting:
                    self._drain([b])
        return ids

    def _neighbourhood(self, p):
        return [b for b, _ in self._nearest(self.cent[p], self.reassign_neighbors + 2)]

    def _local_moves(self, p, cands):
        ids, _ = self._live_entries(p)
        cands = [t for t in cands if t != p and self._is_live(t)]
        moves = []
        if not cands or len(ids) == 0:
            return moves
        V = self.raw[ids.astype(np.int64)]
        D = _seq_matrix(self.metric, V, self.cent[[p] + cands])
        best = np.argmin(D[:, 1:], axis=1)
        better = D[np.arange(len(ids)), 1 + best] < D[:, 0]
        for j in np.nonzero(better)[0]:
            moves.append((int(ids[j]), cands[int(best[j])]))
        return moves

    def _drain(self, queue):
        while queue:
            b = queue.pop()
            if not self._is_live(b):
                continue
            if self._len(b) >= self.max_posting:
                self._split(b, queue)
            else:
                self._relocate(b, self._local_moves(b, self._neighbourhood(b)), queue)

    def _relocate(self, frm, moves, queue):
        if not moves:
            return
        mv = dict(moves)
        ids, codes = self._live_entries(frm)
        keep = np.array([int(i) not in mv for i in ids], dtype=bool)
        self._rewrite(frm, ids[keep], codes[keep])
        dest, added = [], {}  # target of each moved entry; entries pushed to a slot so far
        for id_ in ids[~keep]:
            t = mv[int(id_)]
            if not (self._is_live(t) and self._len(t) + added.get(t, 0) < 2 * self.max_posting):
                if frm not in queue:
                    queue.insert(0, frm)
                if self._is_live(t):
                    queue.append(t)
                t = frm
            dest.append(t)
            added[t] = added.get(t, 0) + 1
            if self._len(t) + added[t] >= self.max_posting:
                queue.append(t)
        moved = codes[~keep]
        if self.codec.residual and len(dest):  # re-encoded against the target's centroid, one call per target
            moved = moved.copy()
            dest_a = np.array(dest)
            for t in np.unique(dest_a):
                sel = np.nonzero(dest_a == t)[0]
                moved[sel] = self.codec.encode(self.raw[ids[~keep][sel].astype(np.int64)], self.cent[t])
        for id_, code, t in zip(ids[~keep], moved, dest):
            self._push(t, int(id_), code)

    def _split(self, b, queue):
        # Splits converge for metric distances; a score such as 1 - dot on
        # unnormalised data routes every vector to the largest centroid and
        # keeps splitting, which shows as more postings than vectors.
        if int(self.live_b.sum()) > max(64, self.next_id):
            raise RuntimeError("Index error: SPFresh splits did not converge "
                               "(more postings than vectors; a non-metric score on unnormalised data?)")
        ids, codes = self._live_entries(b)
        if len(ids) < 2:
            self._rewrite(b, ids, codes)
            return
        vs = self.raw[ids.astype(np.int64)]
        c1, c2, side = kmeans2(vs, self.metric)
        self._free_posting(b)
        nb = [self._new_posting(c1), self._new_posting(c2)]
        if self.codec.residual:  # re-encoded against the new centroids, one call per new posting
            codes = codes.copy()
            for sd in (False, True):
                sel = np.nonzero(side == sd)[0]
                if len(sel):
                    codes[sel] = self.codec.encode(vs[sel], self.cent[nb[int(sd)]])
        for id_, code, sd in zip(ids, codes, side):
            self._push(nb[int(sd)], int(id_), code)
        around = sorted({q for p in nb for q in self._neighbourhood(p)})
        for p in nb:
            self._relocate(p, self._local_moves(p, around), queue)
        for q in around:
            if q in nb or not self._is_live(q):
                continue
            self._relocate(q, self._local_moves(q, nb), queue)
        for p in nb:
            if self._len(p) >= self.max_posting:
                queue.append(p)

    @locked
    def delete(self, ids):
        """SPFresh::delete (src/spfresh.rs:863-871): tombstones."""
        for i in ids:
            i = int(i)
            if i < self.next_id and i not in self.deleted:
                self.deleted.add(i)
                self.live -= 1
        self._sync()

    @locked
    def is_deleted(self, id):  # noqa: A002
        return int(id) in self.deleted

    @locked
    def get_vector(self, id):  # noqa: A002
        id = int(id)  # noqa: A001
        return None if id >= self.next_id or id in self.deleted else self.raw[id].tolist()

    @locked
    def gc(self):
        """Inner::gc (src/spfresh.rs:613-643): purge tombstones, merge small postings."""
        self.epoch += 1
        queue = []
        for b in range(len(self.live_b)):
            if not self._is_live(b):
                continue
            ids, codes = self._live_entries(b)
            if len(ids) < self.min_posting and int(self.live_b.sum()) > 1:
                self._free_posting(b)
                for id_, code in zip(ids, codes):
                    v = self.raw[int(id_)]
                    nn = self._nearest(v, 1)
                    t = nn[0][0] if nn else int(np.nonzero(self.live_b)[0][0])
                    if self.codec.residual:
                        code = self._encode(v, t)
                    self._push(t, int(id_), code)
                    if self._len(t) >= self.max_posting:
                        queue.append(t)
                        self._drain(queue)
            elif len(ids) != self._len(b):
                self._rewrite(b, ids, codes)
        self._drain(queue)
        self._sync()

    @locked
    def compact(self):
        """SPFresh::compact (src/spfresh.rs:645-669, 916-918).  The reference
        rebuilds its centroid graph over the live postings and renumbers
        their centroid ids 0..n-1, because it routes a query by a beam search
        over that graph.  This mirror routes exactly, over the live
        centroids on the device, and numbers live postings consecutively at
        every save, so no routing state goes stale: compact publishes the
        pending posting changes to the device and leaves results unchanged."""
        self._sync()

    @locked
    def stats(self):
        sizes = [self._len(b) for b in range(len(self.live_b)) if self._is_live(b)]
        return {"live": self.live, "deleted": len(self.deleted), "postings": int(self.live_b.sum()),
                "max_posting": max(sizes) if sizes else 0}

    # ------------------------------------------------------------ persistence
    @staticmethod
    def open(path, metric="l2", device=0):
        """SPFresh::open (src/spfresh.rs:819-850) of the files SPFresh::save wrote:
        `{path}.spf` (metadata), `.postings` (blocks), `.vectors` (raw rows) and
        `.centroids` (the centroid graph; checked, not used -- routing here is exact)."""
        from . import formats as F

        if metric not in _METRICS:
            raise ValueError(f"unknown metric: {metric}")
        meta = F.parse_spf(_read(f"{path}.spf"))
        F.check_incremental_header(_read(f"{path}.centroids"))
        kind, qp = _codec_params(meta.quantizer)
        cfg, d, nb = meta.cfg, meta.dim, len(meta.block_cid)
        s = SPFresh(d, metric, kind, qp, cfg.rerank_size, max(cfg.max_posting_size, 2), cfg.min_posting_size,
                    cfg.reassign_neighbors, cfg.probe_ratio, device)
        s.centroid_beam = cfg.centroid_beam
        block = F.spf_block_bytes(cfg, meta.quantizer, d)
        posts = F.parse_postings(_read(f"{path}.postings"), nb, block, s.codec.size)
        live = meta.block_cid != np.uint64(F.SPF_FREE)
        s.cent = np.zeros((nb, d), dtype=np.float32)
        for b in np.nonzero(live)[0]:
            s.cent[b] = meta.block_centroid[b]
        s.live_b = live
        s.ids = [ids if live[b] else ids[:0] for b, (ids, _) in enumerate(posts)]
        s.codes = [codes if live[b] else codes[:0] for b, (_, codes) in enumerate(posts)]
        s.free = [(int(b), 0) for b in np.nonzero(~live)[0]]  # src/spfresh.rs:834-840
        n = meta.next_id
        for b, ids in enumerate(s.ids):
            if len(ids) and int(ids.max()) >= n:
                raise RuntimeError(f"Index error: block {b} holds id {int(ids.max())} >= next_id {n}")
        if meta.deleted.size and int(meta.deleted.max()) >= n:
            raise RuntimeError(f"Index error: deleted id {int(meta.deleted.max())} >= next_id {n}")
        raw = np.frombuffer(_read(f"{path}.vectors"), dtype="<f4")
        if raw.size < n * d:
            raise RuntimeError(f"Index error: vectors file holds {raw.size // max(d, 1)} rows, next_id {n}")
        s.raw = raw[: n * d].reshape(n, d).astype(np.float32)
        s.next_id, s.deleted, s.live = n, {int(i) for i in meta.deleted}, int(meta.live)
        s.path = path
        s._dirty = set(range(nb))
        s._sync()
        return s

    @locked
    def save(self, path=None):
        """SPFresh::save (src/spfresh.rs:852-859): the four files SPFresh::open reads.

        Live postings get consecutive centroid ids in a delta-only
        IncrementalDiskANN (the layout the reference's centroid graph has
        before any merge), whose graph is a Vamana graph over the centroids
        built on the GPU (IncrementalConfig's delta parameters: degree 32,
        beam 64, alpha 1.2, src/incremental.rs:31-43)."""
        from . import formats as F

        path = path or self.path
        if path is None:
            raise RuntimeError("Index error: no path to save to")
        q = _quantizer_state(self)
        cfg = F.SPFreshConfig(self.max_posting, self.min_posting, self.probe_ratio, self.rerank_size,
                              self.reassign_neighbors, self.centroid_beam)
        nb = len(self.live_b)
        live_blocks = np.nonzero(self.live_b)[0]
        cid = np.full(nb, F.SPF_FREE, dtype=np.uint64)
        cid[live_blocks] = np.uint64(F.DELTA_ID_OFFSET) + np.arange(len(live_blocks), dtype=np.uint64)
        cents = [self.cent[b].astype(np.float32) if self.live_b[b] else np.zeros(0, np.float32) for b in range(nb)]
        meta = F.SPFreshMeta(self.dim, cfg, q, cid, cents, self.next_id,
                             np.array(sorted(self.deleted), dtype=np.uint64), self.live)
        block = F.spf_block_bytes(cfg, q, self.dim)
        F._write(f"{path}.postings", F.postings_bytes(list(zip(self.ids, self.codes)), block, self.codec.size))
        rows = np.zeros((max(self.next_id, 1024), self.dim), dtype="<f4")
        rows[: self.next_id] = self.raw[: self.next_id]
        F._write(f"{path}.vectors", rows.tobytes())
        C_ = np.ascontiguousarray(self.cent[live_blocks], dtype=np.float32)
        graph, ep = _centroid_graph(C_, self.metric_name, self.device)
        F._write(f"{path}.centroids", F.incremental_bytes(C_.reshape(-1, self.dim), graph, ep, 32))
        F._write(f"{path}.spf", F.spf_bytes(meta))
        self.path = path

    # ------------------------------------------------------------ device side
    def host_arrays(self, nblocks=None):
        """Posting slots as the flat arrays of DgSpfreshDesc."""
        nb = nblocks or max(len(self.live_b), 1)
        cent = np.zeros((nb, self.dim), dtype=np.float32)
        cent[: len(self.cent)] = self.cent
        live = np.zeros(nb, dtype=np.uint8)
        live[: len(self.live_b)] = self.live_b
        lens = np.zeros(nb, dtype=np.uint32)
        ids = np.full((nb, self.cap), np.uint64(_lib.PAD64), dtype=np.uint64)
        codes = np.zeros((nb, self.cap, self.codec.size), dtype=np.uint8)
        for b in range(len(self.live_b)):
            n = self._len(b)
            lens[b] = n
            ids[b, :n] = self.ids[b]
            codes[b, :n] = self.codes[b]
        return cent, live, lens, ids, codes

    def _block_arrays(self, blocks):
        """The slots in `blocks` (all below len(live_b)) as DgSpfreshDesc rows."""
        m = len(blocks)
        cent = np.ascontiguousarray(self.cent[blocks], dtype=np.float32)
        live = np.ascontiguousarray(self.live_b[blocks], dtype=np.uint8)
        lens = np.zeros(m, dtype=np.uint32)
        ids = np.full((m, self.cap), np.uint64(_lib.PAD64), dtype=np.uint64)
        codes = np.zeros((m, self.cap, self.codec.size), dtype=np.uint8)
        for j, b in enumerate(blocks):
            n = self._len(b)
            lens[j] = n
            ids[j, :n] = self.ids[b]
            codes[j, :n] = self.codes[b]
        return cent, live, lens, ids, codes

    def _sync(self):
        if self.device is None:  # host-only instance (update logic without a GPU mirror)
            return
        if self._h is None or len(self.live_b) > self._dev_blocks or self.next_id > self._dev_ids:
            self._create_device()
            return
        if self._dirty:
            blocks = np.array(sorted(self._dirty), dtype=np.uint32)
            cent, live, lens, ids, codes = self._block_arrays(blocks)
            check(lib().dg_spfresh_update_blocks(self._h, ptr(blocks), len(blocks), ptr(cent), ptr(live), ptr(lens),
                                                 ptr(ids), ptr(codes)))
            self._dirty.clear()
            self._cent_dirty.clear()
        if self.next_id > self._raw_synced:
            rows = np.ascontiguousarray(self.raw[self._raw_synced:self.next_id])
            check(lib().dg_spfresh_put_raw(self._h, self._raw_synced, ptr(rows), len(rows)))
            self._raw_synced = self.next_id
        new_del = self.deleted - self._del_synced
        if new_del:
            arr = np.array(sorted(new_del), dtype=np.uint64)
            check(lib().dg_spfresh_set_deleted(self._h, ptr(arr), len(arr), 1))
            self._del_synced |= new_del

    def _create_device(self):
        if self._h is not None:
            lib().dg_spfresh_destroy(self._h)
            self._h = None
        # room for new postings without re-creating the mirror: x2 for small
        # indexes, +25 % for large ones (host staging is slots x cap x code bytes)
        n_slots = len(self.live_b)
        nb = max(2 * n_slots if n_slots < 4096 else n_slots + n_slots // 4, 16)
        id_cap = max(2 * self.next_id, 1024)
        cent, live, lens, ids, codes = self.host_arrays(nb)
        raw = np.ascontiguousarray(self.raw[: self.next_id])
        dele = np.zeros(id_cap, dtype=np.uint8)
        for i in self.deleted:
            dele[i] = 1
        d = _lib.SpfreshDesc()
        d.dim, d.metric, d.device, d.num_blocks, d.block_cap = self.dim, self.metric, self.device, nb, self.cap
        keep = [cent, live, lens, ids, codes, raw, dele]
        d.centroids, d.block_live, d.block_len = ptr(cent), ptr(live), ptr(lens)
        d.entry_ids, d.entry_codes, d.code_size = ptr(ids), ptr(codes), self.codec.size
        kinds = {None: _lib.Q_NONE, "f16": _lib.Q_F16, "int8": _lib.Q_INT8, "pq": _lib.Q_PQ, "rabitq": _lib.Q_RABITQ}
        d.quantizer = kinds[self.codec.kind]
        if self.codec.kind == "pq":
            cb = np.ascontiguousarray(self.codec.p["codebooks"], dtype=np.float32)
            keep.append(cb)
            d.pq_M, d.pq_K, d.pq_codebooks = cb.shape[0], cb.shape[1], ptr(cb)
        if self.codec.kind == "int8":
            d.int8_scale, d.int8_offset = self.codec.p["scale"], self.codec.p["offset"]
        if self.codec.kind == "rabitq":
            sg = np.ascontiguousarray(self.codec.p["signs"], dtype=np.float32)
            keep.append(sg)
            d.rq_padded, d.rq_signs = self.codec.p["padded"], ptr(sg)
        d.id_capacity, d.num_raw, d.raw, d.deleted = id_cap, self.next_id, ptr(raw), ptr(dele)
        h = C.c_void_p()
        check(lib().dg_spfresh_create(C.byref(d), C.byref(h)))
        self._h = h
        self._dev_blocks, self._dev_ids = nb, id_cap
        self._dirty.clear()
        self._cent_dirty.clear()
        self._raw_synced = self.next_id
        self._del_synced = set(self.deleted)

    @locked
    def close(self):
        if self._h is not None:
            lib().dg_spfresh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------------- search
    @locked
    def search_arrays(self, queries, k=10, n_probe=8, stream=None):
        """Batched search: numpy in -> numpy out (ids u64, dists f32, counts u32),
        or CUDA tensors in -> tensors out."""
        if self._h is None:
            raise RuntimeError("Index error: this SPFresh instance has no device mirror (device=None)")
        dev = hasattr(queries, "data_ptr") and getattr(queries, "is_cuda", False)
        p = _lib.SpfreshParams()
        p.k, p.nprobe, p.rerank_size, p.probe_ratio = k, n_probe, self.rerank_size, self.probe_ratio
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
            out = (torch.empty((nq, k), dtype=torch.int64, device=Q.device),
                   torch.empty((nq, k), dtype=torch.float32, device=Q.device),
                   torch.empty((nq,), dtype=torch.int32, device=Q.device))
            p.flags = _lib.FLAG_DEVICE_PTRS | _lib.FLAG_STREAM
            p.stream = stream if stream is not None else torch.cuda.current_stream(Q.device).cuda_stream
        else:
            Q = _lib.query_rows(queries, self.dim)
            nq = Q.shape[0]
            out = (np.empty((nq, k), dtype=np.uint64), np.empty((nq, k), dtype=np.float32),
                   np.empty(nq, dtype=np.uint32))
        if Q.shape[1] != self.dim:
            raise ValueError(f"Query dim {Q.shape[1]} != index dim {self.dim}")
        check(lib().dg_spfresh_search_batch(self._h, C.byref(p), ptr(Q), nq, ptr(out[0]), ptr(out[1]),
                                            ptr(out[2])))
        return out

    def search_with_dists(self, query, k=10, n_probe=8):
        ids, ds, cnt = self.search_arrays(np.asarray(query, dtype=np.float32).reshape(1, -1), k, n_probe)
        return [(int(ids[0, j]), float(ds[0, j])) for j in range(int(cnt[0]))]

    def search(self, query, k=10, n_probe=8):
        return [i for i, _ in self.search_with_dists(query, k, n_probe)]

    def search_batch(self, queries, k=10, n_probe=8):
        ids, ds, cnt = self.search_arrays(queries, k, n_probe)
        return [ids[i, : cnt[i]].astype(np.int64).tolist() for i in range(len(cnt))]



def _read(path):
    from . import formats as F

    try:
        with open(path, "rb") as f:
            return f.read()
    except OSError as e:
        raise F.io_error(e) from None


def _codec_params(q):
    """(codec kind, params) of a saved QuantizerState (None = raw f32 rows)."""
    if q is None:
        return None, {}
    if q.kind == "pq":
        return "pq", {"codebooks": q.codebooks.reshape(q.num_subspaces, q.num_centroids, q.subspace_dim)}
    if q.kind == "int8":
        return "int8", {"scale": q.scale, "offset": q.offset}
    if q.kind == "rabitq":
        return "rabitq", {"padded": q.padded, "signs": q.signs, "centroid": q.centroid}
    return "f16", {}


def _quantizer_state(s):
    from . import formats as F

    k, p = s.codec.kind, s.codec.p
    if k is None:
        return None
    if k == "pq":
        cb = np.asarray(p["codebooks"], dtype=np.float32)
        M, K, ds = cb.shape
        return F.QuantizerState("pq", s.dim, M, K, ds, codebooks=cb.reshape(-1))
    if k == "int8":
        return F.QuantizerState("int8", s.dim, scale=float(p["scale"]), offset=float(p["offset"]))
    if k == "rabitq":
        cen = p.get("centroid")
        if cen is None:  # RaBitQ::train's centroid: the mean row (src/rabitq.rs:78-90)
            cen = (s.raw[: s.next_id].astype(np.float64).sum(0) / max(s.next_id, 1)).astype(np.float32)
        return F.QuantizerState("rabitq", s.dim, padded=int(p["padded"]), centroid=np.asarray(cen, np.float32),
                                signs=np.asarray(p["signs"], dtype=np.float32))
    return F.QuantizerState("f16", s.dim)


def _centroid_graph(C_, metric, device):
    """Adjacency lists (local indexes) and entry point over the live centroids."""
    n = len(C_)
    if n == 0:
        return [], None
    if n == 1:
        return [[]], 0
    if device is not None:
        import pydiskann_b200 as dg

        adj, med = dg.build_graph(C_, max_degree=min(32, n - 1), build_beam_width=64, alpha=1.2,
                                  metric=metric, device=device)
        return [row[row != _lib.PAD].tolist() for row in np.asarray(adj)], int(med)
    # host-only instance: exact nearest-centroid lists
    graph = []
    for c0 in range(0, n, 1024):
        D = _seq_matrix(_METRICS[metric], C_[c0:c0 + 1024], C_)
        for i in range(len(D)):
            D[i, c0 + i] = np.inf
        graph += np.argsort(D, axis=1, kind="stable")[:, : min(32, n - 1)].tolist()
    return graph, 0
