"""Restatement of the reference's SPFresh update path (TEST INFRASTRUCTURE ONLY).

The checker of the posting lists the product maintains on the host
(pydiskann_b200/spfresh.py): only tests/ use it, never the product.  It follows
diskann-rs src/spfresh.rs statement by statement:
  Inner::alloc / new_posting / free_posting      :380-415
  Inner::insert (CHUNK = 4096 vectors per epoch)  :416-476
  Inner::local_moves / neighbourhood / drain     :488-520
  Inner::relocate                                 :522-558
  Inner::split + kmeans2                          :560-611, :122-162
  Inner::gc                                       :613-643
Codes come from the oracle's C encoders (int8 / PQ); raw postings store the
f32 bytes of the vector.

Refinements shared with the product, each fixed here so that a comparison is
exact:
  * nearest() is brute force over the live postings at every size (the
    reference switches to its centroid graph above 4096 postings, a graph it
    builds non-deterministically) and orders equal distances by slot;
  * every distance is the f32 sum of squared differences in coordinate order,
    the oracle's metric_eval (the reference's distances come from numkong,
    f32 with an order no test pins).
"""
from __future__ import annotations

import numpy as np

CHUNK = 4096  # src/spfresh.rs:21


def _l2_direct(v, C):
    """f32 coordinate-order squared L2 of v against every row of C."""
    C = np.asarray(C, dtype=np.float32)
    v = np.asarray(v, dtype=np.float32)
    acc = np.zeros(len(C), dtype=np.float32)
    for i in range(C.shape[1]):
        t = v[i] - C[:, i]
        acc = acc + t * t
    return acc


def _l2_matrix(V, C):
    """_l2_direct for every row of V: f32 [len(V), len(C)]."""
    V = np.asarray(V, dtype=np.float32)
    C = np.asarray(C, dtype=np.float32)
    out = np.zeros((len(V), len(C)), dtype=np.float32)
    for i in range(V.shape[1] if len(V) else 0):
        t = V[:, i, None] - C[None, :, i]
        out = out + t * t
    return out


class RefSpfresh:
    """Posting slots of the reference's Inner: per slot a live flag, a centroid
    and an ordered list of (id, code) entries; a free list of (slot, epoch)."""

    def __init__(self, dim, max_posting, min_posting=16, reassign_neighbors=16, encode=None):
        self.dim = dim
        self.max_posting = max(max_posting, 2)
        self.min_posting = min_posting
        self.reassign_neighbors = reassign_neighbors
        self.encode_rows = encode or (lambda V: np.ascontiguousarray(V, dtype=np.float32).view(np.uint8))
        self.live_slot = []      # block_cid != FREE
        self.centroid = []       # block_centroid
        self.entries = []        # per slot: list of (id, bytes)
        self.free = []           # [(slot, epoch)]
        self.created = []
        self.epoch = 1
        self.raw = []            # raw f32 vectors by id
        self.next_id = 0
        self.deleted = set()
        self.live = 0

    # ---------------------------------------------------------------- slots
    def n_live(self):
        return sum(self.live_slot)

    def is_live(self, b):
        return 0 <= b < len(self.live_slot) and self.live_slot[b]

    def live_entries(self, b):
        return [(i, c) for i, c in self.entries[b] if i not in self.deleted]

    def alloc(self):
        for i, (b, e) in enumerate(self.free):
            if e < self.epoch:
                last = self.free.pop()
                if i < len(self.free):
                    self.free[i] = last
                return b
        self.live_slot.append(False)
        self.centroid.append(None)
        self.entries.append([])
        return len(self.live_slot) - 1

    def new_posting(self, centroid):
        b = self.alloc()
        self.live_slot[b] = True
        self.centroid[b] = np.asarray(centroid, dtype=np.float32).copy()
        self.created.append(b)
        self.entries[b] = []
        return b

    def free_posting(self, b):
        self.live_slot[b] = False
        self.centroid[b] = None
        self.entries[b] = []
        self.free.append((b, self.epoch))

    def push(self, b, id_, code):
        self.entries[b].append((id_, code))

    def encode(self, v):
        return bytes(self.encode_rows(np.asarray(v, dtype=np.float32).reshape(1, -1))[0])

    # -------------------------------------------------------------- routing
    def live_slots(self):
        return [b for b in range(len(self.live_slot)) if self.live_slot[b]]

    def nearest(self, v, n):
        live = self.live_slots()
        if not live:
            return []
        d = _l2_direct(v, np.stack([self.centroid[b] for b in live]))
        order = sorted(range(len(live)), key=lambda i: (d[i], live[i]))[:n]
        return [(live[i], float(d[i])) for i in order]

    def dist(self, v, b):
        return float(_l2_direct(v, self.centroid[b][None])[0])

    # --------------------------------------------------------------- insert
    def insert(self, vectors):
        vectors = np.asarray(vectors, dtype=np.float32)
        ids = list(range(self.next_id, self.next_id + len(vectors)))
        self.raw.extend(v.copy() for v in vectors)
        self.next_id += len(vectors)
        self.live += len(vectors)
        queue = []
        for c0 in range(0, len(vectors), CHUNK):
            chunk = vectors[c0:c0 + CHUNK]
            self.epoch += 1
            self.created = []
            live = self.live_slots()
            if live:
                D = _l2_matrix(chunk, np.stack([self.centroid[b] for b in live]))
                targets = [live[int(j)] for j in np.argmin(D, axis=1)]
            else:
                targets = [None] * len(chunk)
            for j, v in enumerate(chunk):
                id_ = ids[c0 + j]
                t = targets[j]
                best = (t, self.dist(v, t)) if t is not None and self.is_live(t) else None
                if best is None:
                    nn = self.nearest(v, 1)
                    best = nn[0] if nn else None
                for c in list(self.created):
                    if self.is_live(c):
                        d = self.dist(v, c)
                        if best is None or d < best[1]:
                            best = (c, d)
                b = best[0] if best is not None else self.new_posting(v)
                self.push(b, id_, self.encode(v))
                if len(self.entries[b]) >= self.max_posting:
                    queue.append(b)
                    self.drain(queue)
        return ids

    def delete(self, ids):
        for i in ids:
            i = int(i)
            if i < self.next_id and i not in self.deleted:
                self.deleted.add(i)
                self.live -= 1

    # ------------------------------------------------------------- maintain
    def local_moves(self, p, cands):
        ents = self.live_entries(p)
        cands = [t for t in cands if t != p and self.is_live(t)]
        if not cands or not ents:
            return []
        V = np.stack([self.raw[i] for i, _ in ents])
        D = _l2_matrix(V, np.stack([self.centroid[p]] + [self.centroid[t] for t in cands]))
        moves = []
        for r, (id_, _) in enumerate(ents):
            j = int(np.argmin(D[r, 1:]))  # the first minimum, as Iterator::min_by
            if D[r, 1 + j] < D[r, 0]:
                moves.append((id_, cands[j]))
        return moves

    def neighbourhood(self, p):
        return [b for b, _ in self.nearest(self.centroid[p], self.reassign_neighbors + 2)]

    def drain(self, queue):
        while queue:
            b = queue.pop()
            if not self.is_live(b):
                continue
            if len(self.entries[b]) >= self.max_posting:
                self.split(b, queue)
            else:
                self.relocate(b, self.local_moves(b, self.neighbourhood(b)), queue)

    def relocate(self, frm, moves, queue):
        if not moves:
            return
        target = {}
        for id_, t in moves:
            target.setdefault(id_, t)
        ents = self.live_entries(frm)
        moved = [e for e in ents if e[0] in target]
        self.entries[frm] = [e for e in ents if e[0] not in target]
        for id_, code in moved:
            t = target[id_]
            if not (self.is_live(t) and len(self.entries[t]) < 2 * self.max_posting):
                if frm not in queue:
                    queue.insert(0, frm)
                if self.is_live(t):
                    queue.append(t)
                t = frm
            self.push(t, id_, code)
            if len(self.entries[t]) >= self.max_posting:
                queue.append(t)

    @staticmethod
    def kmeans2(vs):
        n = len(vs)

        def means(side):
            out = []
            for k in (False, True):
                sel = vs[side == k]
                cnt = max(len(sel), 1)
                out.append((sel.sum(0, dtype=np.float32) / np.float32(cnt)).astype(np.float32))
            return out

        far = 0
        if n > 1:
            d0 = _l2_direct(vs[0], vs[1:])
            far = 1 + int(np.argmax(d0))
        c = [vs[0].copy(), vs[far].copy()]
        side = np.zeros(n, dtype=bool)
        for _ in range(5):
            side = _l2_direct(c[1], vs) < _l2_direct(c[0], vs)
            if side.all() or not side.any():
                break
            c = means(side)
        if side.all() or not side.any():
            side = np.arange(n) >= n // 2
            c = means(side)
        return c[0], c[1], side

    def split(self, b, queue):
        ents = self.live_entries(b)
        if len(ents) < 2:
            self.entries[b] = ents
            return
        vs = np.stack([self.raw[i] for i, _ in ents])
        c1, c2, side = self.kmeans2(vs)
        self.free_posting(b)
        nb = [self.new_posting(c1), self.new_posting(c2)]
        for (id_, code), s in zip(ents, side):
            self.push(nb[int(s)], id_, code)
        around = sorted({q for p in nb for q in self.neighbourhood(p)})
        for p in nb:
            self.relocate(p, self.local_moves(p, around), queue)
        for q in around:
            if q in nb or not self.is_live(q):
                continue
            self.relocate(q, self.local_moves(q, nb), queue)
        for p in nb:
            if len(self.entries[p]) >= self.max_posting:
                queue.append(p)

    def gc(self):
        self.epoch += 1
        queue = []
        for b in range(len(self.live_slot)):
            if not self.is_live(b):
                continue
            ents = self.live_entries(b)
            if len(ents) < self.min_posting and self.n_live() > 1:
                self.free_posting(b)
                for id_, code in ents:
                    nn = self.nearest(self.raw[id_], 1)
                    t = nn[0][0] if nn else self.live_slots()[0]
                    self.push(t, id_, code)
                    if len(self.entries[t]) >= self.max_posting:
                        queue.append(t)
                        self.drain(queue)
            elif len(ents) != len(self.entries[b]):
                self.entries[b] = ents
        self.drain(queue)

    # --------------------------------------------------------------- export
    def postings(self):
        """{slot: (ids u64[], codes u8[n, code])} of the live slots."""
        out = {}
        for b in self.live_slots():
            ids = np.array([i for i, _ in self.entries[b]], dtype=np.uint64)
            codes = np.frombuffer(b"".join(c for _, c in self.entries[b]), dtype=np.uint8)
            out[b] = (ids, codes.reshape(len(ids), -1) if len(ids) else codes.reshape(0, 0))
        return out
