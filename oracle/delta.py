"""Pure-Python restatement of IncrementalDiskANN's delta layer (test infrastructure).

Follows DeltaLayer::add_vectors (diskann-rs src/incremental.rs:114-166),
compute_medoid (:168-193), find_and_prune_neighbors (:195-209),
greedy_search_internal (:211-280) and robust_prune (src/lib.rs:977-1034,
alpha 1.2), in loops, for the small graphs the CPU tests build.  Equal
distances are ordered by id (the reference leaves them in heap order).
Distances are float32 sums; the tests use integer-valued vectors, so every
sum is exact in any order.
"""
from __future__ import annotations

import heapq

import numpy as np

L2SQ, L2, COSINE, DOT = 0, 1, 2, 3


def _dist(metric, a, b):
    if metric in (L2SQ, L2):
        t = (a - b).astype(np.float32)
        s = np.float32((t * t).sum(dtype=np.float32))
        return np.float32(np.sqrt(s)) if metric == L2 else s
    if metric == DOT:
        return np.float32(1.0) - np.float32((a * b).sum(dtype=np.float32))
    raise ValueError("the restatement covers l2 / euclidean / dot")


class DeltaLayer:
    def __init__(self, dim, max_degree=32, metric=L2SQ):
        self.dim, self.R, self.metric = dim, max_degree, metric
        self.vectors: list[np.ndarray] = []
        self.graph: list[list[int]] = []
        self.entry = None

    def d(self, a, b):
        return float(_dist(self.metric, self.vectors[a], self.vectors[b]))

    def greedy(self, q, start, beam):
        visited = {start}
        s = (float(_dist(self.metric, q, self.vectors[start])), start)
        frontier = [s]
        res = [(-s[0], -s[1])]  # max-heap of (d, id) through negation
        while frontier:
            best = frontier[0]
            if len(res) >= beam and best[0] >= -res[0][0]:
                break
            heapq.heappop(frontier)
            for nb in self.graph[best[1]] if best[1] < len(self.graph) else []:
                if nb in visited:
                    continue
                visited.add(nb)
                if nb >= len(self.vectors):
                    continue
                c = (float(_dist(self.metric, q, self.vectors[nb])), nb)
                worst = (-res[0][0], -res[0][1])
                if len(res) < beam:
                    heapq.heappush(res, (-c[0], -c[1]))
                    heapq.heappush(frontier, c)
                elif c < worst:
                    heapq.heapreplace(res, (-c[0], -c[1]))
                    heapq.heappush(frontier, c)
        return [(-d, -i) for d, i in res]

    def prune(self, node, cands):
        srt = sorted((d, i) for d, i in cands if i != node)
        uniq = []
        for d, i in srt:
            if not uniq or uniq[-1][1] != i:
                uniq.append((d, i))
        n = len(uniq)
        alpha = np.float32(1.2)
        occ = [np.float32(0.0)] * n
        sel = [False] * n
        out = []
        cur = np.float32(1.0)
        while cur <= alpha and len(out) < self.R:
            for i in range(n):
                if len(out) >= self.R:
                    break
                if sel[i] or occ[i] > cur:
                    continue
                sel[i] = True
                out.append(uniq[i][1])
                for j in range(i + 1, n):
                    if sel[j] or occ[j] > alpha:
                        continue
                    djk = np.float32(self.d(uniq[j][1], uniq[i][1]))
                    occ[j] = np.float32(np.inf) if djk == 0 else max(occ[j], np.float32(uniq[j][0]) / djk)
            cur = np.float32(cur * np.float32(1.2))
        for i in range(n):
            if len(out) >= self.R:
                break
            if not sel[i]:
                sel[i] = True
                out.append(uniq[i][1])
        return out

    def medoid(self):
        c = np.zeros(self.dim, dtype=np.float32)
        for v in self.vectors:
            c += v
        c /= np.float32(len(self.vectors))
        ds = [float(_dist(self.metric, c, v)) for v in self.vectors]
        return int(np.argmin(ds))

    def add_vectors(self, X):
        for v in np.asarray(X, dtype=np.float32):
            node = len(self.vectors)
            self.vectors.append(v.copy())
            self.graph.append([])
            if node > 0:
                beam = max(self.R * 2, 16)
                if self.entry is not None:
                    cands = self.greedy(v, self.entry, beam)
                else:
                    cands = [(self.d(node, i), i) for i in range(node)]
                nbrs = self.prune(node, cands)
                self.graph[node] = list(nbrs)
                for nb in nbrs:
                    if node in self.graph[nb]:
                        continue
                    if len(self.graph[nb]) < self.R:
                        self.graph[nb].append(node)
                    else:
                        pool = [(self.d(nb, c), c) for c in self.graph[nb] + [node]]
                        self.graph[nb] = self.prune(nb, pool)
            if self.entry is None:
                self.entry = 0
        if len(self.vectors) > 1:
            self.entry = self.medoid()

    def adjacency(self):
        A = np.full((len(self.graph), self.R), 0xFFFFFFFF, dtype=np.uint32)
        for i, row in enumerate(self.graph):
            A[i, : len(row)] = row
        return A
