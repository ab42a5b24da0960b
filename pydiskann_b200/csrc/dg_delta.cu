// dg_delta.cu -- the delta layer of a base + delta (incremental) index.
//
// DeltaLayer::add_vectors (diskann-rs src/incremental.rs:114-166) inserts one
// vector at a time: a greedy search from the entry point over the graph the
// previous inserts wrote (:211-280), robust_prune of what it found
// (src/lib.rs:977-1034, alpha 1.2), then back-edges, re-pruning a neighbour
// whose list is full.  Each insert depends on the graph the previous one left,
// so this runs on the host; the searches over base + delta run on the GPU.
//
// Ties: candidates are ordered by (distance, id) wherever the reference
// leaves equal distances in heap order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <queue>
#include <string>
#include <vector>

#include "dg_common.cuh"

namespace {

struct Cand {
  float d;
  uint32_t id;
};
inline bool lex_less(const Cand &a, const Cand &b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }
struct Less {
  bool operator()(const Cand &a, const Cand &b) const { return lex_less(a, b); }
};
struct Greater {
  bool operator()(const Cand &a, const Cand &b) const { return lex_less(b, a); }
};

// src/metric.rs:16-39 with a left-to-right f32 accumulation.
float metric_eval(int32_t metric, const float *a, const float *b, uint32_t d) {
  if (metric == DG_L2SQ || metric == DG_L2) {
    float acc = 0.0f;
    for (uint32_t i = 0; i < d; ++i) {
      const float t = a[i] - b[i];
      acc += t * t;
    }
    return metric == DG_L2 ? std::sqrt(acc) : acc;
  }
  if (metric == DG_DOT) {
    float acc = 0.0f;
    for (uint32_t i = 0; i < d; ++i) acc += a[i] * b[i];
    return 1.0f - acc;
  }
  float ab = 0.0f, aa = 0.0f, bb = 0.0f;  // 1 - cos; 0 for two zero vectors, 1 when orthogonal
  for (uint32_t i = 0; i < d; ++i) {
    ab += a[i] * b[i];
    aa += a[i] * a[i];
    bb += b[i] * b[i];
  }
  if (aa == 0.0f && bb == 0.0f) return 0.0f;
  if (ab == 0.0f) return 1.0f;
  const float r = 1.0f - ab / (std::sqrt(aa) * std::sqrt(bb));
  return r > 0.0f ? r : 0.0f;
}

struct Delta {
  const float *X;
  uint32_t dim, R;
  int32_t metric;
  uint32_t *adj;
  uint64_t n;  // rows inserted so far
  std::vector<uint32_t> stamp;
  uint32_t epoch = 0;

  const float *row(uint64_t i) const { return X + i * dim; }
  uint32_t degree(uint64_t i) const {
    const uint32_t *r = adj + i * R;
    uint32_t c = 0;
    while (c < R && r[c] != DG_PAD) ++c;
    return c;
  }
  float dist(uint64_t a, uint64_t b) const { return metric_eval(metric, row(a), row(b), dim); }

  // greedy_search_internal (src/incremental.rs:211-280)
  std::vector<Cand> greedy(const float *q, uint32_t start, uint32_t beam) {
    if (++epoch == 0) {
      std::fill(stamp.begin(), stamp.end(), 0u);
      epoch = 1;
    }
    std::priority_queue<Cand, std::vector<Cand>, Greater> frontier;  // top = min
    std::priority_queue<Cand, std::vector<Cand>, Less> res;         // top = max
    const Cand s{metric_eval(metric, q, row(start), dim), start};
    frontier.push(s);
    res.push(s);
    stamp[start] = epoch;
    while (!frontier.empty()) {
      const Cand best = frontier.top();
      if (res.size() >= beam && best.d >= res.top().d) break;
      frontier.pop();
      const uint32_t *r = adj + (uint64_t)best.id * R;
      for (uint32_t j = 0; j < R && r[j] != DG_PAD; ++j) {
        const uint32_t nb = r[j];
        if (stamp[nb] == epoch) continue;
        stamp[nb] = epoch;
        if (nb >= n) continue;
        const Cand c{metric_eval(metric, q, row(nb), dim), nb};
        if (res.size() < beam) {
          res.push(c);
          frontier.push(c);
        } else if (lex_less(c, res.top())) {
          res.pop();
          res.push(c);
          frontier.push(c);
        }
      }
    }
    std::vector<Cand> out;
    out.reserve(res.size());
    while (!res.empty()) {
      out.push_back(res.top());
      res.pop();
    }
    return out;
  }

  // robust_prune (src/lib.rs:977-1034) with alpha 1.2; writes the row of `node`
  void prune(uint32_t node, std::vector<Cand> cands) {
    std::vector<Cand> sorted;
    sorted.reserve(cands.size());
    for (const Cand &c : cands)
      if (c.id != node) sorted.push_back(c);
    std::sort(sorted.begin(), sorted.end(), lex_less);
    sorted.erase(std::unique(sorted.begin(), sorted.end(), [](const Cand &a, const Cand &b) { return a.id == b.id; }),
                 sorted.end());
    const size_t m = sorted.size();
    const float alpha = 1.2f;
    std::vector<float> occlude(m, 0.0f);
    std::vector<char> selected(m, 0);
    std::vector<uint32_t> pruned;
    pruned.reserve(std::min<size_t>(R, m));
    float cur = 1.0f;
    while (cur <= alpha && pruned.size() < R) {
      for (size_t i = 0; i < m; ++i) {
        if (pruned.size() >= R) break;
        if (selected[i] || occlude[i] > cur) continue;
        selected[i] = 1;
        pruned.push_back(sorted[i].id);
        for (size_t j = i + 1; j < m; ++j) {
          if (selected[j] || occlude[j] > alpha) continue;
          const float djk = dist(sorted[j].id, sorted[i].id);
          occlude[j] = djk == 0.0f ? INFINITY : std::max(occlude[j], sorted[j].d / djk);
        }
      }
      cur *= 1.2f;
    }
    for (size_t i = 0; i < m && pruned.size() < R; ++i)
      if (!selected[i]) {
        selected[i] = 1;
        pruned.push_back(sorted[i].id);
      }
    uint32_t *r = adj + (uint64_t)node * R;
    for (uint32_t j = 0; j < R; ++j) r[j] = j < pruned.size() ? pruned[j] : DG_PAD;
  }

  // compute_medoid (src/incremental.rs:168-193): nearest row to the mean row
  uint32_t medoid() const {
    std::vector<float> c(dim, 0.0f);
    for (uint64_t i = 0; i < n; ++i)
      for (uint32_t j = 0; j < dim; ++j) c[j] += row(i)[j];
    for (uint32_t j = 0; j < dim; ++j) c[j] /= (float)n;
    uint32_t best = 0;
    float bd = 0.0f;
    for (uint64_t i = 0; i < n; ++i) {
      const float d = metric_eval(metric, c.data(), row(i), dim);
      if (i == 0 || d < bd) {
        bd = d;
        best = (uint32_t)i;
      }
    }
    return best;
  }
};

}  // namespace

extern "C" DgStatus dg_delta_insert(const float *vectors, uint32_t dim, int32_t metric, uint32_t max_degree,
                                    uint32_t *adjacency, uint64_t n_old, uint64_t n_new, int64_t *entry_point) {
  if (!vectors || !adjacency || !entry_point) return dg::fail(DG_EINVAL, "null argument");
  if (dim == 0 || max_degree == 0) return dg::fail(DG_EINVAL, "dim and max_degree must be >= 1");
  if (metric < DG_L2SQ || metric > DG_DOT) return dg::fail(DG_EINVAL, "unknown metric");
  if (n_old + n_new >= (1ull << 31)) return dg::fail(DG_EINVAL, "delta rows must stay below 2^31");
  if (*entry_point < -1 || (*entry_point >= 0 && (uint64_t)*entry_point >= n_old))
    return dg::fail(DG_EINVAL, "entry point out of range");
  for (uint64_t i = 0; i < n_old * max_degree; ++i)
    if (adjacency[i] != DG_PAD && adjacency[i] >= n_old) return dg::fail(DG_EINVAL, "delta graph id out of range");
  Delta g{vectors, dim, max_degree, metric, adjacency, n_old, std::vector<uint32_t>(n_old + n_new, 0u)};
  int64_t entry = *entry_point;
  const uint32_t beam = std::max<uint32_t>(max_degree * 2, 16);  // find_and_prune_neighbors, :199-209
  for (uint64_t t = 0; t < n_new; ++t) {
    const uint32_t node = (uint32_t)(n_old + t);
    g.n = (uint64_t)node + 1;
    uint32_t *r = adjacency + (uint64_t)node * max_degree;
    for (uint32_t j = 0; j < max_degree; ++j) r[j] = DG_PAD;
    if (node > 0) {
      std::vector<Cand> cands;
      if (entry >= 0) {
        cands = g.greedy(g.row(node), (uint32_t)entry, beam);
      } else {
        for (uint32_t i = 0; i < node; ++i) cands.push_back({g.dist(node, i), i});
      }
      g.prune(node, cands);
      std::vector<uint32_t> nbrs(r, r + g.degree(node));
      for (uint32_t nb : nbrs) {
        uint32_t *nr = adjacency + (uint64_t)nb * max_degree;
        const uint32_t deg = g.degree(nb);
        if (std::find(nr, nr + deg, node) != nr + deg) continue;
        if (deg < max_degree) {
          nr[deg] = node;
        } else {
          std::vector<Cand> pool;
          pool.reserve(deg + 1);
          for (uint32_t j = 0; j < deg; ++j) pool.push_back({g.dist(nb, nr[j]), nr[j]});
          pool.push_back({g.dist(nb, node), node});
          g.prune(nb, pool);
        }
      }
    }
    if (entry < 0) entry = 0;
  }
  if (g.n > 1) entry = g.medoid();
  *entry_point = entry;
  return DG_OK;
}
