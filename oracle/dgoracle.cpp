// dgoracle.cpp -- CPU restatement of the diskann-rs search hot path.
//
// TEST INFRASTRUCTURE ONLY: the correctness oracle for pydiskann_b200's CUDA
// kernels (see dgoracle.h for the contract and the list of refinements).
// Built with -ffp-contract=off so that every float expression rounds exactly
// as written; the CUDA kernels use explicit round-to-nearest intrinsics for the
// same expressions, which makes codes, lookup tables and estimator values
// bit-identical between the two.
#include "dgoracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <queue>
#include <unordered_set>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();

struct Cand {
  float d;
  uint32_t id;
};

// Candidate order (src/lib.rs:101-122 orders by distance only and leaves
// equal distances in heap order); the oracle refines ties by node id.
inline bool lex_less(const Cand &a, const Cand &b) {
  return a.d < b.d || (a.d == b.d && a.id < b.id);
}
struct LexLess {
  bool operator()(const Cand &a, const Cand &b) const { return lex_less(a, b); }
};
struct LexGreater {
  bool operator()(const Cand &a, const Cand &b) const { return lex_less(b, a); }
};

// ---------------------------------------------------------------- distances
// numkong (third-party, not in the reference tree) supplies these kernels;
// the oracle fixes a sequential left-to-right f32 accumulation.
float l2sq(const float *a, const float *b, uint32_t d) {
  float acc = 0.0f;
  for (uint32_t i = 0; i < d; ++i) {
    float t = a[i] - b[i];
    acc += t * t;
  }
  return acc;
}
float dot(const float *a, const float *b, uint32_t d) {
  float acc = 0.0f;
  for (uint32_t i = 0; i < d; ++i) acc += a[i] * b[i];
  return acc;
}
// numkong angular: 1 - cos(a, b), 0 for two zero vectors, 1 when orthogonal.
float angular(const float *a, const float *b, uint32_t d) {
  float ab = 0.0f, aa = 0.0f, bb = 0.0f;
  for (uint32_t i = 0; i < d; ++i) {
    ab += a[i] * b[i];
    aa += a[i] * a[i];
    bb += b[i] * b[i];
  }
  if (aa == 0.0f && bb == 0.0f) return 0.0f;
  if (ab == 0.0f) return 1.0f;
  float r = 1.0f - ab / (std::sqrt(aa) * std::sqrt(bb));
  return r > 0.0f ? r : 0.0f;
}
// src/metric.rs:16-39 (DistL2 = sqrt of sqeuclidean, DistDot = 1 - dot).
float metric_eval(int32_t metric, const float *a, const float *b, uint32_t d) {
  switch (metric) {
    case DGO_L2SQ: return l2sq(a, b, d);
    case DGO_L2: return std::sqrt(l2sq(a, b, d));
    case DGO_COSINE: return angular(a, b, d);
    default: return 1.0f - dot(a, b, d);
  }
}

// ------------------------------------------------------------ random stream
inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline uint64_t rand4(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
  return mix64(mix64(mix64(seed + a) + b) + c);
}
inline uint64_t range_of(uint64_t r, uint64_t n) {
  return (uint64_t)(((unsigned __int128)r * (unsigned __int128)n) >> 64);
}

// --------------------------------------------------------------- beam search
// Restates beam_search (src/lib.rs:198-303): best-first search with a
// frontier min-heap, a working max-heap `w` of `working` entries, a visited
// set, and for filtered search the insertion-sorted result list, the
// early-termination factor and the iteration cap.
struct BeamCfg {
  bool filtered = false;
  uint32_t expanded = 0;
  uint64_t max_iter = UINT64_MAX;
  float early = kInf;
};

template <class DistFn, class NbrFn, class FiltFn>
void beam_search(const uint32_t *seeds, uint32_t nseeds, uint32_t beam, uint32_t k, DistFn dist,
                 NbrFn nbrs, FiltFn filt, const BeamCfg &cfg, std::vector<Cand> &out,
                 uint32_t *stats, bool return_all_w = false) {
  const uint32_t working = cfg.filtered ? cfg.expanded : beam;
  std::unordered_set<uint32_t> visited;
  std::priority_queue<Cand, std::vector<Cand>, LexGreater> frontier;  // top = min
  std::priority_queue<Cand, std::vector<Cand>, LexLess> w;            // top = max
  std::vector<Cand> results;
  uint32_t n_exp = 0, n_dist = 0;

  auto result_insert = [&](const Cand &c) {
    size_t pos = results.size();
    for (size_t i = 0; i < results.size(); ++i)
      if (lex_less(c, results[i])) { pos = i; break; }
    if (pos < k) {
      results.insert(results.begin() + pos, c);
      if (results.size() > k) results.pop_back();
    }
  };

  for (uint32_t s = 0; s < nseeds; ++s) {
    uint32_t sid = seeds[s];
    if (!visited.insert(sid).second) continue;
    float d = dist(sid);
    ++n_dist;
    Cand c{d, sid};
    frontier.push(c);
    w.push(c);
    if (cfg.filtered && filt(sid)) results.push_back(c);
  }
  if (cfg.filtered) {
    std::sort(results.begin(), results.end(), lex_less);
    if (results.size() > k) results.resize(k);
  }

  uint64_t iterations = 0;
  std::vector<uint32_t> nb;
  while (!frontier.empty()) {
    Cand best = frontier.top();
    ++iterations;
    if (iterations > cfg.max_iter) break;
    if (cfg.filtered && results.size() >= k && k > 0) {
      float worst = results.back().d;
      if (std::isfinite(cfg.early) && worst >= 0.0f &&
          best.d > worst * std::max(cfg.early, 1.0f))
        break;
    }
    if (w.size() >= working && !w.empty()) {
      if (best.d >= w.top().d) break;
    }
    frontier.pop();
    ++n_exp;
    nbrs(best.id, nb);
    for (uint32_t id : nb) {
      if (!visited.insert(id).second) continue;
      float d = dist(id);
      ++n_dist;
      Cand c{d, id};
      if (w.size() < working) {
        w.push(c);
        frontier.push(c);
      } else if (lex_less(c, w.top())) {
        w.pop();
        w.push(c);
        frontier.push(c);
      }
      if (cfg.filtered && filt(id)) result_insert(c);
    }
  }
  if (stats) {
    stats[0] = n_exp;
    stats[1] = n_dist;
  }
  if (cfg.filtered) {
    out = results;
    return;
  }
  out.clear();
  out.reserve(w.size());
  while (!w.empty()) {
    out.push_back(w.top());
    w.pop();
  }
  std::sort(out.begin(), out.end(), lex_less);
  if (!return_all_w && out.size() > k) out.resize(k);
}

struct AdjNbrs {
  const uint32_t *adj;
  uint32_t R;
  void operator()(uint32_t id, std::vector<uint32_t> &nb) const {
    nb.clear();
    const uint32_t *row = adj + (uint64_t)id * R;
    for (uint32_t j = 0; j < R; ++j)
      if (row[j] != DGO_PAD) nb.push_back(row[j]);
  }
};

// ------------------------------------------------------------- robust prune
// src/lib.rs:977-1034 (strict alpha=1 pass, relaxed passes up to alpha, then
// backfill).  Input need not be sorted; it is sorted by (dist, id), which is
// what the reference's stable sort by distance yields on its id-sorted input.
template <class PairDist>
void robust_prune(uint32_t node, std::vector<Cand> cands, uint32_t R, float alpha,
                  PairDist pdist, std::vector<uint32_t> &pruned) {
  std::vector<Cand> sorted;
  sorted.reserve(cands.size());
  for (auto &c : cands)
    if (c.id != node) sorted.push_back(c);
  std::sort(sorted.begin(), sorted.end(), lex_less);
  sorted.erase(std::unique(sorted.begin(), sorted.end(),
                           [](const Cand &a, const Cand &b) { return a.id == b.id; }),
               sorted.end());
  const size_t n = sorted.size();
  alpha = std::max(alpha, 1.0f);
  std::vector<float> occlude(n, 0.0f);
  std::vector<char> selected(n, 0);
  pruned.clear();
  float cur_alpha = 1.0f;
  while (cur_alpha <= alpha && pruned.size() < R) {
    for (size_t i = 0; i < n; ++i) {
      if (pruned.size() >= R) break;
      if (selected[i] || occlude[i] > cur_alpha) continue;
      selected[i] = 1;
      pruned.push_back(sorted[i].id);
      for (size_t j = i + 1; j < n; ++j) {
        if (selected[j] || occlude[j] > alpha) continue;
        float djk = pdist(sorted[j].id, sorted[i].id);
        occlude[j] = djk == 0.0f ? kInf : std::max(occlude[j], sorted[j].d / djk);
      }
    }
    cur_alpha = cur_alpha * 1.2f;
  }
  for (size_t i = 0; i < n; ++i) {
    if (pruned.size() >= R) break;
    if (!selected[i]) {
      selected[i] = 1;
      pruned.push_back(sorted[i].id);
    }
  }
}

// ------------------------------------------------------------------- filter
// Postfix form of Filter::matches (src/filtered.rs:120-135); a missing field
// never matches, And of nothing is true, Or of nothing is false.
bool filter_eval(const DgoFilterOp *prog, uint32_t nops, const uint64_t *pool,
                 const uint64_t *labels, uint32_t nf) {
  if (nops == 0) return true;
  bool stack[64];
  int sp = 0;
  for (uint32_t i = 0; i < nops; ++i) {
    const DgoFilterOp &o = prog[i];
    bool v = false;
    switch (o.op) {
      case DGO_F_TRUE: v = true; break;
      case DGO_F_EQ: v = o.field < nf && labels[o.field] == o.a; break;
      case DGO_F_IN:
        if (o.field < nf) {
          uint64_t x = labels[o.field];
          for (uint64_t t = 0; t < o.b; ++t)
            if (pool[o.a + t] == x) { v = true; break; }
        }
        break;
      case DGO_F_LT: v = o.field < nf && labels[o.field] < o.a; break;
      case DGO_F_GT: v = o.field < nf && labels[o.field] > o.a; break;
      case DGO_F_RANGE: v = o.field < nf && labels[o.field] >= o.a && labels[o.field] <= o.b; break;
      case DGO_F_AND:
      case DGO_F_OR: {
        uint32_t c = o.field;
        bool acc = o.op == DGO_F_AND;
        for (uint32_t t = 0; t < c; ++t) {
          bool x = stack[--sp];
          acc = o.op == DGO_F_AND ? (acc && x) : (acc || x);
        }
        v = acc;
        break;
      }
      default: v = false;
    }
    stack[sp++] = v;
  }
  return sp > 0 ? stack[sp - 1] : true;
}

// -------------------------------------------------------------- quantizers
struct PqState {
  uint32_t d, M, K, ds;
  const float *cb;
  const float *centroid(uint32_t m, uint32_t c) const { return cb + ((uint64_t)m * K + c) * ds; }
};

// src/pq.rs:181-198
void pq_lut(const PqState &pq, const float *q, float *lut) {
  for (uint32_t m = 0; m < pq.M; ++m)
    for (uint32_t c = 0; c < pq.K; ++c) lut[m * pq.K + c] = l2sq(q + m * pq.ds, pq.centroid(m, c), pq.ds);
}
// src/pq.rs:202-209 -- sequential f32 sum over subspaces.
float pq_adc(const float *lut, const uint8_t *code, uint32_t M, uint32_t K) {
  float d = 0.0f;
  for (uint32_t m = 0; m < M; ++m) d += lut[m * K + code[m]];
  return d;
}
void pq_decode(const PqState &pq, const uint8_t *code, float *out) {
  for (uint32_t m = 0; m < pq.M; ++m) std::memcpy(out + m * pq.ds, pq.centroid(m, code[m]), pq.ds * 4);
}

// src/sq.rs:208-220: x * (1/scale) + (-offset/scale), rounded to nearest
// (ties to even) and saturated to [0, 255].
uint8_t int8_code(float x, float inv, float beta) {
  float t = x * inv + beta;
  if (!(t == t)) return 0;
  t = std::nearbyint(t);
  if (t < 0.0f) return 0;
  if (t > 255.0f) return 255;
  return (uint8_t)t;
}
void int8_encode_row(const float *x, uint32_t d, float scale, float offset, uint8_t *out) {
  float inv = 1.0f / scale;
  float beta = -offset / scale;
  for (uint32_t i = 0; i < d; ++i) out[i] = int8_code(x[i], inv, beta);
}
// src/sq.rs:168-172: exact integer sum, converted to f32, times scale twice.
float int8_dist(const uint8_t *q, const uint8_t *c, uint32_t d, float scale) {
  uint64_t s = 0;
  for (uint32_t i = 0; i < d; ++i) {
    int t = (int)q[i] - (int)c[i];
    s += (uint64_t)(t * t);
  }
  return (float)s * scale * scale;
}

inline uint16_t f32_to_f16(float x) {
  _Float16 h = (_Float16)x;
  uint16_t u;
  std::memcpy(&u, &h, 2);
  return u;
}
inline float f16_to_f32(uint16_t u) {
  _Float16 h;
  std::memcpy(&h, &u, 2);
  return (float)h;
}
float f16_dist(const uint16_t *q, const uint16_t *c, uint32_t d) {
  float acc = 0.0f;
  for (uint32_t i = 0; i < d; ++i) {
    float t = f16_to_f32(q[i]) - f16_to_f32(c[i]);
    acc += t * t;
  }
  return acc;
}

// RaBitQ (src/rabitq.rs).
void fht(float *v, uint32_t n) {  // :31-43
  for (uint32_t h = 1; h < n; h *= 2)
    for (uint32_t i = 0; i < n; i += 2 * h)
      for (uint32_t j = i; j < i + h; ++j) {
        float x = v[j], y = v[j + h];
        v[j] = x + y;
        v[j + h] = x - y;
      }
}
void rq_rotate(float *v, uint32_t P, const float *signs) {  // :121-126
  for (int r = 0; r < 3; ++r) {
    for (uint32_t i = 0; i < P; ++i) v[i] *= signs[r * P + i];
    fht(v, P);
  }
}
void rq_unrotate(float *v, uint32_t P, const float *signs) {  // :128-133
  for (int r = 2; r >= 0; --r) {
    fht(v, P);
    for (uint32_t i = 0; i < P; ++i) v[i] *= signs[r * P + i];
  }
}
// :136-149 -> (rotated unit residual, norm)
float rq_prep(const float *v, uint32_t d, uint32_t P, const float *cen, const float *signs,
              float *r) {
  for (uint32_t i = 0; i < P; ++i) r[i] = i < d ? v[i] - cen[i] : 0.0f;
  float s = 0.0f;
  for (uint32_t i = 0; i < P; ++i) s += r[i] * r[i];
  float norm = std::sqrt(s);
  if (norm > 0.0f)
    for (uint32_t i = 0; i < P; ++i) r[i] /= norm;
  rq_rotate(r, P, signs);
  return norm;
}
// :240-256
void rq_pack(const float *r, uint32_t P, float norm, uint8_t *code) {
  float ip = 0.0f;
  for (uint32_t c = 0; c < P / 64; ++c) {
    uint64_t w = 0;
    for (uint32_t i = 0; i < 64; ++i) {
      float x = r[c * 64 + i];
      w |= (uint64_t)(x > 0.0f) << i;
      ip += std::fabs(x);
    }
    std::memcpy(code + c * 8, &w, 8);
  }
  ip /= std::sqrt((float)P);
  float fac = ip > 0.0f ? norm / ip : 0.0f;
  float n2 = norm * norm;
  std::memcpy(code + P / 8, &n2, 4);
  std::memcpy(code + P / 8 + 4, &fac, 4);
}
// :157-187
void rq_query(const float *q, uint32_t d, uint32_t P, const float *cen, const float *signs,
              uint64_t *planes, float *k5) {
  std::vector<float> r(P);
  float nq = rq_prep(q, d, P, cen, signs, r.data());
  float lo = std::numeric_limits<float>::max(), hi = std::numeric_limits<float>::lowest();
  for (uint32_t i = 0; i < P; ++i) {
    lo = std::min(lo, r[i]);
    hi = std::max(hi, r[i]);
  }
  const float levels = 15.0f;
  float delta = (hi - lo) / levels;
  float inv = delta > 0.0f ? 1.0f / delta : 0.0f;
  uint32_t words = P / 64;
  std::memset(planes, 0, sizeof(uint64_t) * 4 * words);
  uint32_t sum_u = 0;
  for (uint32_t i = 0; i < P; ++i) {
    float t = std::round((r[i] - lo) * inv);
    uint32_t u = t <= 0.0f ? 0u : (uint32_t)t;
    u = std::min(u, 15u);
    sum_u += u;
    for (uint32_t j = 0; j < 4; ++j)
      if ((u >> j) & 1u) planes[j * words + i / 64] |= 1ull << (i % 64);
  }
  float sd = std::sqrt((float)P);
  k5[0] = nq * nq;
  k5[1] = 2.0f * nq;
  k5[2] = 2.0f * delta / sd;
  k5[3] = 2.0f * lo / sd;
  k5[4] = -(delta * (float)sum_u + (float)P * lo) / sd;
}
void rq_bits(const uint8_t *code, const uint64_t *planes, uint32_t words, uint32_t &S,
             uint32_t &C) {  // :46-58
  S = 0;
  C = 0;
  for (uint32_t i = 0; i < words; ++i) {
    uint64_t b;
    std::memcpy(&b, code + i * 8, 8);
    C += __builtin_popcountll(b);
    S += __builtin_popcountll(b & planes[i]) + (__builtin_popcountll(b & planes[words + i]) << 1) +
         (__builtin_popcountll(b & planes[2 * words + i]) << 2) +
         (__builtin_popcountll(b & planes[3 * words + i]) << 3);
  }
}
float rq_est(const uint64_t *planes, const float *k5, const uint8_t *code, uint32_t P) {  // :191-197
  uint32_t S, C;
  rq_bits(code, planes, P / 64, S, C);
  float n2, fac;
  std::memcpy(&n2, code + P / 8, 4);
  std::memcpy(&fac, code + P / 8 + 4, 4);
  float e = n2 + k5[0] - k5[1] * fac * (k5[2] * (float)S + k5[3] * (float)C + k5[4]);
  return std::fmax(e, 0.0f);
}
void rq_est_bound(const uint64_t *planes, const float *k5, const uint8_t *code, uint32_t P,
                  float &est, float &err) {  // :202-215
  est = rq_est(planes, k5, code, P);
  float n2, fac;
  std::memcpy(&n2, code + P / 8, 4);
  std::memcpy(&fac, code + P / 8 + 4, 4);
  float ip = fac > 0.0f ? std::sqrt(n2) / fac : 0.0f;
  err = ip > 0.0f
            ? k5[1] * fac * 1.9f * std::sqrt(std::fmax(1.0f - ip * ip, 0.0f) / ((float)P - 1.0f))
            : kInf;
}
void rq_decode(const uint8_t *code, uint32_t d, uint32_t P, const float *cen, const float *signs,
               float *out) {  // :224-238
  std::vector<float> r(P);
  float sd = std::sqrt((float)P);
  for (uint32_t c = 0; c < P / 64; ++c) {
    uint64_t b;
    std::memcpy(&b, code + c * 8, 8);
    for (uint32_t i = 0; i < 64; ++i) r[c * 64 + i] = ((b >> i) & 1) ? 1.0f / sd : -1.0f / sd;
  }
  rq_unrotate(r.data(), P, signs);
  float n2;
  std::memcpy(&n2, code + P / 8, 4);
  float norm = std::sqrt(n2);
  for (uint32_t i = 0; i < d; ++i) out[i] = cen[i] + norm * r[i];
}

// Per-query prepared state (src/quantized.rs:57-62,167-174).
// ---------------------------------------------------------------- FP8 e4m3
// OCP 8-bit floating point, E4M3: bias 7, no infinities, 0x7F / 0xFF are NaN,
// largest finite 448 (0x7E), subnormals k * 2^-9.  Positive codes 0x00..0x7E
// are increasing in value, so encoding is a nearest search with ties to the
// even code; anything at or above 448 saturates to 448.
static float e4m3_value(uint32_t c) {  // c in 0..0x7E
  const uint32_t E = c >> 3, f = c & 7u;
  return E == 0 ? std::ldexp((float)f, -9) : std::ldexp(1.0f + (float)f / 8.0f, (int)E - 7);
}
uint8_t e4m3_encode(float x) {
  if (x != x) return 0x7F;
  const uint8_t sign = std::signbit(x) ? 0x80 : 0x00;
  const float a = std::fabs(x);
  if (a >= 448.0f) return sign | 0x7E;
  uint32_t lo = 0, hi = 0x7E;  // largest code with value <= a
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) / 2;
    if (e4m3_value(mid) <= a) lo = mid;
    else hi = mid - 1;
  }
  uint32_t c = lo;
  if (e4m3_value(c) < a) {
    const float dl = a - e4m3_value(c), du = e4m3_value(c + 1) - a;
    if (du < dl || (du == dl && ((c + 1) & 1u) == 0)) c = c + 1;
  }
  return sign | (uint8_t)c;
}
float e4m3_decode(uint8_t c) {
  const float v = e4m3_value(c & 0x7Fu);
  return (c & 0x80u) ? -v : v;
}
float fp8_row(const float *x, uint32_t d, uint8_t *code) {  // -> scale
  float mx = 0.0f;
  for (uint32_t i = 0; i < d; ++i) mx = std::fmax(mx, std::fabs(x[i]));
  const float s = mx > 0.0f ? mx / 448.0f : 1.0f;
  for (uint32_t i = 0; i < d; ++i) code[i] = e4m3_encode(x[i] / s);
  return s;
}

// ---------------------------------------------------------------- BF16
static uint16_t f32_to_bf16(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);  // quiet NaN
  u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest, ties to even
  return (uint16_t)(u >> 16);
}
static float bf16_to_f32(uint16_t h) {
  const uint32_t u = (uint32_t)h << 16;
  float x;
  std::memcpy(&x, &u, 4);
  return x;
}

struct Prepared {
  std::vector<float> lut;
  std::vector<uint8_t> u8;
  std::vector<uint16_t> h;
  std::vector<uint64_t> planes;
  float k5[5];
  std::vector<float> fhi, flo;  // FP8: e4m3 values of the scaled query q' and of 16 (q' - hi)
  float fs = 1.0f, fqq = 0.0f;  // FP8: query scale, |q|^2
};

void prepare(const DgoIndex &I, const float *q, Prepared &p) {
  switch (I.quant) {
    case DGO_Q_PQ: {
      PqState pq{I.d, I.pq_M, I.pq_K, I.d / I.pq_M, I.pq_codebooks};
      p.lut.resize((size_t)I.pq_M * I.pq_K);
      pq_lut(pq, q, p.lut.data());
      break;
    }
    case DGO_Q_INT8:
      p.u8.resize(I.d);
      int8_encode_row(q, I.d, I.int8_scale, I.int8_offset, p.u8.data());
      break;
    case DGO_Q_F16:
      p.h.resize(I.d);
      for (uint32_t i = 0; i < I.d; ++i) p.h[i] = f32_to_f16(q[i]);
      break;
    case DGO_Q_FP8: {
      float mx = 0.0f, qq = 0.0f;
      for (uint32_t i = 0; i < I.d; ++i) {
        mx = std::fmax(mx, std::fabs(q[i]));
        qq += q[i] * q[i];
      }
      p.fs = mx > 0.0f ? mx / 448.0f : 1.0f;
      p.fqq = qq;
      p.fhi.resize(I.d);
      p.flo.resize(I.d);
      for (uint32_t i = 0; i < I.d; ++i) {
        const float v = q[i] / p.fs;
        p.fhi[i] = e4m3_decode(e4m3_encode(v));
        p.flo[i] = e4m3_decode(e4m3_encode((v - p.fhi[i]) * 16.0f));
      }
      break;
    }
    case DGO_Q_RABITQ:
      p.planes.resize(4 * (I.rq_padded / 64));
      rq_query(q, I.d, I.rq_padded, I.rq_centroid, I.rq_signs, p.planes.data(), p.k5);
      break;
  }
}

// src/quantized.rs:13-54: L2/L2Sq use the quantizer's squared estimate (sqrt
// for DistL2); other metrics decode the code and evaluate the metric.
float quantized_distance(const DgoIndex &I, const float *q, uint32_t id, const Prepared &p,
                         std::vector<float> &scratch) {
  const uint8_t *code = I.codes + (uint64_t)id * I.code_size;
  if (I.quant == DGO_Q_FP8) {
    // x = s_x e, q = s_q q': q.x = s_x s_q (e.hi + e.lo / 16), contracted as
    // |q|^2 + |x|^2 - 2 q.x for L2 (FP32 sums in coordinate order)
    const float sx = I.fp8_scale[id];
    float ch = 0.0f, cl = 0.0f, xx = 0.0f;
    for (uint32_t i = 0; i < I.d; ++i) {
      const float e = e4m3_decode(code[i]);
      ch += e * p.fhi[i];
      cl += e * p.flo[i];
      const float xv = sx * e;
      xx += xv * xv;
    }
    const float dot = sx * p.fs * (ch + cl * 0.0625f);
    switch (I.metric) {
      case DGO_L2SQ: return std::fmax(p.fqq + xx - 2.0f * dot, 0.0f);
      case DGO_L2: return std::sqrt(std::fmax(p.fqq + xx - 2.0f * dot, 0.0f));
      case DGO_DOT: return 1.0f - dot;
      default: {
        if (p.fqq == 0.0f && xx == 0.0f) return 0.0f;
        if (dot == 0.0f) return 1.0f;
        const float r = 1.0f - dot / (std::sqrt(p.fqq) * std::sqrt(xx));
        return r > 0.0f ? r : 0.0f;
      }
    }
  }
  if (I.quant == DGO_Q_BF16) {  // the metric of the f32 query against the decoded row
    scratch.resize(I.d);
    for (uint32_t i = 0; i < I.d; ++i) {
      uint16_t u;
      std::memcpy(&u, code + 2 * i, 2);
      scratch[i] = bf16_to_f32(u);
    }
    return metric_eval(I.metric, q, scratch.data(), I.d);
  }
  if (I.metric != DGO_L2SQ && I.metric != DGO_L2) {
    scratch.resize(I.d);
    switch (I.quant) {
      case DGO_Q_PQ: {
        PqState pq{I.d, I.pq_M, I.pq_K, I.d / I.pq_M, I.pq_codebooks};
        pq_decode(pq, code, scratch.data());
        break;
      }
      case DGO_Q_INT8:
        for (uint32_t i = 0; i < I.d; ++i) scratch[i] = (float)code[i] * I.int8_scale + I.int8_offset;
        break;
      case DGO_Q_F16:
        for (uint32_t i = 0; i < I.d; ++i) {
          uint16_t u;
          std::memcpy(&u, code + 2 * i, 2);
          scratch[i] = f16_to_f32(u);
        }
        break;
      case DGO_Q_RABITQ:
        rq_decode(code, I.d, I.rq_padded, I.rq_centroid, I.rq_signs, scratch.data());
        break;
    }
    return metric_eval(I.metric, q, scratch.data(), I.d);
  }
  float d = 0.0f;
  switch (I.quant) {
    case DGO_Q_PQ: d = pq_adc(p.lut.data(), code, I.pq_M, I.pq_K); break;
    case DGO_Q_INT8: d = int8_dist(p.u8.data(), code, I.d, I.int8_scale); break;
    case DGO_Q_F16: d = f16_dist(p.h.data(), (const uint16_t *)code, I.d); break;
    case DGO_Q_RABITQ: d = rq_est(p.planes.data(), p.k5, code, I.rq_padded); break;
  }
  return I.metric == DGO_L2 ? std::sqrt(d) : d;
}

int nthreads_of(int32_t t) {
#ifdef _OPENMP
  return t > 0 ? t : omp_get_max_threads();
#else
  (void)t;
  return 1;
#endif
}

// One query of DiskANN / FilteredDiskANN / QuantizedDiskANN search.
void search_one(const DgoIndex &I, const DgoSearchParams &P, const float *q, uint32_t L,
                std::vector<Cand> &out, uint32_t *stats) {
  const uint32_t k = P.k;
  const bool filt_on = P.filter_nops > 0;
  AdjNbrs nb{I.adjacency, I.R};
  auto allow = [&](uint32_t id) -> bool {
    if (id >= I.n) return false;
    return filter_eval(P.filter, P.filter_nops, P.filter_pool, I.labels + (uint64_t)id * I.num_fields,
                       I.num_fields);
  };
  BeamCfg cfg;
  if (filt_on) {  // src/filtered.rs:35-56, src/quantized.rs:377-397
    cfg.filtered = true;
    cfg.expanded = std::max(L * 4, k * 10);
    cfg.max_iter = (uint64_t)cfg.expanded * 2;
    cfg.early = 1.5f;
  }
  const uint32_t seed = I.medoid;
  if (!P.use_codes) {
    auto dist = [&](uint32_t id) { return metric_eval(I.metric, q, I.vectors + (uint64_t)id * I.d, I.d); };
    beam_search(&seed, 1, L, k, dist, nb, allow, cfg, out, stats);
    return;
  }
  Prepared prep;
  prepare(I, q, prep);
  std::vector<float> scratch;
  auto qdist = [&](uint32_t id) { return quantized_distance(I, q, id, prep, scratch); };
  const uint32_t search_k = P.rerank_size > 0 ? std::max(P.rerank_size, k) : k;
  beam_search(&seed, 1, L, search_k, qdist, nb, allow, cfg, out, stats);
  if (P.rerank_size > 0) {  // src/quantized.rs:110-121: exact distances, stable sort
    for (auto &c : out) c.d = metric_eval(I.metric, q, I.vectors + (uint64_t)c.id * I.d, I.d);
    std::stable_sort(out.begin(), out.end(), [](const Cand &a, const Cand &b) { return a.d < b.d; });
    if (out.size() > k) out.resize(k);
  }
}

}  // namespace

// ======================================================================= C API
extern "C" {

float dgo_distance(int32_t metric, const float *a, const float *b, uint32_t d) {
  return metric_eval(metric, a, b, d);
}

uint64_t dgo_rand(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) { return rand4(seed, a, b, c); }

// src/lib.rs:748-768: vector closest to the centroid.  The centroid is
// summed in f64 and rounded once, and distances are taken in f64, so the
// choice does not depend on a summation order; ties pick the lowest index.
uint32_t dgo_medoid(const float *X, uint64_t n, uint32_t d, int32_t metric) {
  std::vector<double> acc(d, 0.0);
  for (uint64_t i = 0; i < n; ++i)
    for (uint32_t j = 0; j < d; ++j) acc[j] += (double)X[i * d + j];
  std::vector<float> c(d);
  for (uint32_t j = 0; j < d; ++j) c[j] = (float)(acc[j] / (double)n);
  double best = std::numeric_limits<double>::infinity();
  uint32_t bi = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const float *x = X + i * d;
    double v;
    if (metric == DGO_L2SQ || metric == DGO_L2) {
      double s = 0.0;
      for (uint32_t j = 0; j < d; ++j) {
        double t = (double)c[j] - (double)x[j];
        s += t * t;
      }
      v = s;
    } else {
      double ab = 0.0, aa = 0.0, bb = 0.0;
      for (uint32_t j = 0; j < d; ++j) {
        ab += (double)c[j] * (double)x[j];
        aa += (double)c[j] * (double)c[j];
        bb += (double)x[j] * (double)x[j];
      }
      if (metric == DGO_COSINE)
        v = (aa == 0.0 || bb == 0.0) ? 1.0 : 1.0 - ab / (std::sqrt(aa) * std::sqrt(bb));
      else
        v = 1.0 - ab;
    }
    if (v < best) {
      best = v;
      bi = (uint32_t)i;
    }
  }
  return bi;
}

int dgo_robust_prune(uint32_t node, const uint32_t *cand_ids, const float *cand_d, uint32_t nc,
                     const float *X, uint32_t d, int32_t metric, uint32_t R, float alpha,
                     uint32_t *out) {
  std::vector<Cand> c(nc);
  for (uint32_t i = 0; i < nc; ++i) c[i] = Cand{cand_d[i], cand_ids[i]};
  std::vector<uint32_t> pruned;
  robust_prune(node, c, R, alpha,
               [&](uint32_t a, uint32_t b) {
                 return metric_eval(metric, X + (uint64_t)a * d, X + (uint64_t)b * d, d);
               },
               pruned);
  for (size_t i = 0; i < pruned.size(); ++i) out[i] = pruned[i];
  return (int)pruned.size();
}

// src/lib.rs:774-917 with the counter-based random stream:
//   bootstrap draw t of node i   -> rand(seed, 0, i, t)
//   extra search seed e of node u in pass p -> rand(seed, p + 1, u, e)
// The per-pass visit shuffle of the reference is omitted: every node reads the
// previous pass's snapshot and the symmetrised pools are id-sorted, so the
// visit order does not influence the result.
int dgo_build_vamana(const float *X, uint64_t n, uint32_t d, int32_t metric, uint32_t R,
                     uint32_t Lb, float alpha, uint64_t seed, uint32_t medoid, uint32_t *adj,
                     int32_t nthreads) {
  if (n == 0 || R == 0) return -1;
  const int nt = nthreads_of(nthreads);
  std::vector<std::vector<uint32_t>> graph(n);
  const uint64_t target = std::min<uint64_t>(std::max<uint32_t>(R / 2, 2u), n - 1);
  for (uint64_t i = 0; i < n; ++i) {
    std::vector<uint32_t> &g = graph[i];
    uint64_t t = 0;
    while (g.size() < target) {
      uint32_t x = (uint32_t)range_of(rand4(seed, 0, i, t++), n);
      if (x == i) continue;
      if (std::find(g.begin(), g.end(), x) != g.end()) continue;
      g.push_back(x);
    }
  }
  auto vec = [&](uint64_t i) { return X + i * d; };
  auto pdist = [&](uint32_t a, uint32_t b) { return metric_eval(metric, vec(a), vec(b), d); };
  for (uint32_t pass = 0; pass < 2; ++pass) {
    std::vector<std::vector<uint32_t>> ng(n);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
    for (int64_t ui = 0; ui < (int64_t)n; ++ui) {
      const uint32_t u = (uint32_t)ui;
      std::vector<Cand> cands;
      for (uint32_t nb : graph[u]) cands.push_back(Cand{metric_eval(metric, vec(u), vec(nb), d), nb});
      uint32_t seeds[3] = {medoid, (uint32_t)range_of(rand4(seed, pass + 1, u, 0), n),
                           (uint32_t)range_of(rand4(seed, pass + 1, u, 1), n)};
      // greedy_search (src/lib.rs:921-973): the same loop as beam_search,
      // returning the whole working set.
      struct SnapNbrs {
        const std::vector<std::vector<uint32_t>> *g;
        void operator()(uint32_t id, std::vector<uint32_t> &nb) const { nb = (*g)[id]; }
      } sn{&graph};
      auto qd = [&](uint32_t id) { return metric_eval(metric, vec(u), vec(id), d); };
      auto none = [](uint32_t) { return true; };
      std::vector<Cand> part;
      for (uint32_t s = 0; s < 3; ++s) {
        beam_search(&seeds[s], 1, Lb, Lb, qd, sn, none, BeamCfg(), part, nullptr, true);
        cands.insert(cands.end(), part.begin(), part.end());
      }
      std::sort(cands.begin(), cands.end(), [](const Cand &a, const Cand &b) { return a.id < b.id; });
      std::vector<Cand> dedup;
      for (auto &c : cands) {
        if (!dedup.empty() && dedup.back().id == c.id) {
          if (c.d < dedup.back().d) dedup.back().d = c.d;
        } else {
          dedup.push_back(c);
        }
      }
      robust_prune(u, dedup, R, alpha, pdist, ng[u]);
    }
    std::vector<std::vector<uint32_t>> incoming(n);
    for (uint64_t u = 0; u < n; ++u)
      for (uint32_t v : ng[u]) incoming[v].push_back((uint32_t)u);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
    for (int64_t ui = 0; ui < (int64_t)n; ++ui) {
      const uint32_t u = (uint32_t)ui;
      std::vector<uint32_t> ids(ng[u]);
      ids.insert(ids.end(), incoming[u].begin(), incoming[u].end());
      std::sort(ids.begin(), ids.end());
      ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
      std::vector<Cand> pool;
      for (uint32_t id : ids)
        if (id != u) pool.push_back(Cand{metric_eval(metric, vec(u), vec(id), d), id});
      std::vector<uint32_t> pr;
      robust_prune(u, pool, R, alpha, pdist, pr);
      graph[u] = pr;
    }
  }
  for (uint64_t u = 0; u < n; ++u) {
    uint32_t *row = adj + u * R;
    for (uint32_t j = 0; j < R; ++j) row[j] = j < graph[u].size() ? graph[u][j] : DGO_PAD;
  }
  return 0;
}

int dgo_beam_search_table(const uint32_t *adj, uint32_t R, const float *node_dist,
                          const uint8_t *allow, const uint32_t *seeds, uint32_t nseeds,
                          uint32_t L, uint32_t k, int32_t filtered, uint32_t expanded,
                          uint32_t max_iter, float early_factor, uint32_t *out_ids,
                          float *out_d, uint32_t *out_n) {
  BeamCfg cfg;
  if (filtered) {
    cfg.filtered = true;
    cfg.expanded = expanded;
    cfg.max_iter = max_iter;
    cfg.early = early_factor;
  }
  std::vector<Cand> out;
  beam_search(seeds, nseeds, L, k, [&](uint32_t id) { return node_dist[id]; }, AdjNbrs{adj, R},
              [&](uint32_t id) { return allow ? allow[id] != 0 : true; }, cfg, out, nullptr);
  for (size_t i = 0; i < out.size(); ++i) {
    out_ids[i] = out[i].id;
    out_d[i] = out[i].d;
  }
  *out_n = (uint32_t)out.size();
  return 0;
}

int dgo_search_batch(const DgoIndex *idx, const DgoSearchParams *p, const float *Q, uint32_t nq,
                     const uint32_t *per_query_L, uint32_t *out_ids, float *out_d,
                     uint32_t *out_cnt, uint32_t *stats, int32_t nthreads) {
  const int nt = nthreads_of(nthreads);
  const uint32_t k = p->k;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int64_t qi = 0; qi < (int64_t)nq; ++qi) {
    std::vector<Cand> out;
    uint32_t L = per_query_L ? per_query_L[qi] : p->beam_width;
    uint32_t st[2] = {0, 0};
    search_one(*idx, *p, Q + (uint64_t)qi * idx->d, L, out, st);
    for (uint32_t j = 0; j < k; ++j) {
      out_ids[qi * k + j] = j < out.size() ? out[j].id : DGO_PAD;
      out_d[qi * k + j] = j < out.size() ? out[j].d : kInf;
    }
    out_cnt[qi] = (uint32_t)std::min<size_t>(out.size(), k);
    if (stats) {
      stats[2 * qi] = st[0];
      stats[2 * qi + 1] = st[1];
    }
  }
  return 0;
}

int dgo_incremental_search_batch(const DgoIndex *idx, const DgoSearchParams *p, const uint32_t *seeds,
                                 uint32_t nseeds, const uint8_t *dead, uint64_t ntomb, uint64_t code_limit,
                                 const float *Q, uint32_t nq, uint32_t *out_ids, float *out_d, uint32_t *out_cnt,
                                 int32_t nthreads) {
  const DgoIndex &I = *idx;
  const uint32_t k = p->k, L = p->beam_width;
  const bool labeled = p->filter_nops > 0;
  // a label filter searches exact distances (search_filtered_with_dists ignores the quantizer)
  const bool codes = p->use_codes && !labeled;
  const uint32_t search_k = codes && p->rerank_size > 0 ? std::max(p->rerank_size, k) : k;
  BeamCfg cfg;
  if (labeled) {  // search_filtered_with_dists (src/incremental.rs:1048-1062)
    cfg.filtered = true;
    cfg.expanded = std::max(L * 4, k * 10);
    cfg.max_iter = (uint64_t)cfg.expanded * 2;
    cfg.early = 1.5f;
  } else if (ntomb > 0) {  // tombstone_config (src/incremental.rs:505-516)
    cfg.filtered = true;
    cfg.expanded = std::max<uint64_t>((uint64_t)L * 2, search_k + std::min<uint64_t>(ntomb, L));
    cfg.max_iter = (uint64_t)cfg.expanded * 2;
    cfg.early = 1.5f;
  }
  const int nt = nthreads_of(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int64_t qi = 0; qi < (int64_t)nq; ++qi) {
    const float *q = Q + (uint64_t)qi * I.d;
    // UnifiedView::is_live (:463-470), and the label filter when one is given
    auto allow = [&](uint32_t id) -> bool {
      if (id >= I.n || (dead && dead[id])) return false;
      return !labeled || filter_eval(p->filter, p->filter_nops, p->filter_pool,
                                     I.labels + (uint64_t)id * I.num_fields, I.num_fields);
    };
    auto exact = [&](uint32_t id) { return metric_eval(I.metric, q, I.vectors + (uint64_t)id * I.d, I.d); };
    std::vector<Cand> out;
    if (codes) {
      Prepared prep;
      prepare(I, q, prep);
      std::vector<float> scratch;
      auto dist = [&](uint32_t id) {
        return id < code_limit ? quantized_distance(I, q, id, prep, scratch) : exact(id);
      };
      if (nseeds) beam_search(seeds, nseeds, L, search_k, dist, AdjNbrs{I.adjacency, I.R}, allow, cfg, out, nullptr);
      if (p->rerank_size > 0) {  // :972-981: exact distances, sorted, truncated to k
        for (auto &c : out) c.d = exact(c.id);
        std::stable_sort(out.begin(), out.end(), [](const Cand &a, const Cand &b) { return a.d < b.d; });
        if (out.size() > k) out.resize(k);
      }
    } else if (nseeds) {
      beam_search(seeds, nseeds, L, k, exact, AdjNbrs{I.adjacency, I.R}, allow, cfg, out, nullptr);
    }
    for (uint32_t j = 0; j < k; ++j) {
      out_ids[qi * k + j] = j < out.size() ? out[j].id : DGO_PAD;
      out_d[qi * k + j] = j < out.size() ? out[j].d : kInf;
    }
    out_cnt[qi] = (uint32_t)std::min<size_t>(out.size(), k);
  }
  return 0;
}

int dgo_filter_matches(const DgoFilterOp *prog, uint32_t nops, const uint64_t *pool,
                       const uint64_t *labels, uint32_t num_fields) {
  return filter_eval(prog, nops, pool, labels, num_fields) ? 1 : 0;
}

// src/pq.rs:122-149: argmin over centroids with strict '<' (first index wins).
void dgo_pq_encode(const float *X, uint64_t n, uint32_t d, uint32_t M, uint32_t K,
                   const float *cb, uint8_t *codes, int32_t nthreads) {
  PqState pq{d, M, K, d / M, cb};
  const int nt = nthreads_of(nthreads);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    for (uint32_t m = 0; m < M; ++m) {
      const float *sub = X + (uint64_t)i * d + m * pq.ds;
      float best = std::numeric_limits<float>::max();
      uint32_t bc = 0;
      for (uint32_t c = 0; c < K; ++c) {
        float dd = l2sq(sub, pq.centroid(m, c), pq.ds);
        if (dd < best) {
          best = dd;
          bc = c;
        }
      }
      codes[(uint64_t)i * M + m] = (uint8_t)bc;
    }
  }
}
void dgo_pq_lut(const float *q, uint32_t d, uint32_t M, uint32_t K, const float *cb, float *lut) {
  PqState pq{d, M, K, d / M, cb};
  pq_lut(pq, q, lut);
}
float dgo_pq_adc(const float *lut, const uint8_t *code, uint32_t M, uint32_t K) {
  return pq_adc(lut, code, M, K);
}

// src/sq.rs:128-157: one global (min, max) pair.
void dgo_int8_train(const float *X, uint64_t n, uint32_t d, float *scale, float *offset) {
  float lo = std::numeric_limits<float>::max(), hi = std::numeric_limits<float>::lowest();
  for (uint64_t i = 0; i < n * d; ++i) {
    lo = std::min(lo, X[i]);
    hi = std::max(hi, X[i]);
  }
  float range = hi - lo;
  *scale = std::fabs(range) < std::numeric_limits<float>::epsilon() ? 1.0f : range / 255.0f;
  *offset = lo;
}
void dgo_int8_encode(const float *X, uint64_t n, uint32_t d, float scale, float offset,
                     uint8_t *codes) {
  for (uint64_t i = 0; i < n; ++i) int8_encode_row(X + i * d, d, scale, offset, codes + i * d);
}
float dgo_int8_distance(const uint8_t *q, const uint8_t *c, uint32_t d, float scale) {
  return int8_dist(q, c, d, scale);
}
void dgo_f16_encode(const float *X, uint64_t n, uint32_t d, uint16_t *codes) {
  for (uint64_t i = 0; i < n * d; ++i) codes[i] = f32_to_f16(X[i]);
}
float dgo_f16_distance(const uint16_t *q, const uint16_t *c, uint32_t d) { return f16_dist(q, c, d); }
void dgo_bf16_encode(const float *X, uint64_t n, uint32_t d, uint16_t *codes) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)(n * d); ++i) codes[i] = f32_to_bf16(X[i]);
}
uint8_t dgo_e4m3_encode(float x) { return e4m3_encode(x); }
float dgo_e4m3_decode(uint8_t c) { return e4m3_decode(c); }
void dgo_fp8_encode(const float *X, uint64_t n, uint32_t d, uint8_t *codes, float *scales) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)n; ++r) scales[r] = fp8_row(X + r * d, d, codes + r * d);
}


uint32_t dgo_rabitq_padded(uint32_t d) {  // src/rabitq.rs:83
  uint32_t p = 1;
  uint32_t m = std::max(d, 64u);
  while (p < m) p <<= 1;
  return p;
}
void dgo_rabitq_encode(const float *X, uint64_t n, uint32_t d, uint32_t P, const float *cen,
                       const float *signs, uint8_t *codes) {
  std::vector<float> r(P);
  for (uint64_t i = 0; i < n; ++i) {
    float norm = rq_prep(X + i * d, d, P, cen, signs, r.data());
    rq_pack(r.data(), P, norm, codes + i * (P / 8 + 8));
  }
}
void dgo_rabitq_query(const float *q, uint32_t d, uint32_t P, const float *cen, const float *signs,
                      uint64_t *planes, float *k5) {
  rq_query(q, d, P, cen, signs, planes, k5);
}
float dgo_rabitq_distance(const uint64_t *planes, const float *k5, const uint8_t *code, uint32_t P) {
  return rq_est(planes, k5, code, P);
}
void dgo_rabitq_distance_with_bound(const uint64_t *planes, const float *k5, const uint8_t *code,
                                    uint32_t P, float *est, float *err) {
  rq_est_bound(planes, k5, code, P, *est, *err);
}
void dgo_rabitq_decode(const uint8_t *code, uint32_t d, uint32_t P, const float *cen,
                       const float *signs, float *out) {
  rq_decode(code, d, P, cen, signs, out);
}

// SPFresh search (src/spfresh.rs:671-770) with brute-force posting routing
// (src/spfresh.rs:358-378 below its 4096-posting threshold, applied at every
// size here).
int dgo_spfresh_search_batch(const DgoSpfresh *s, const float *Q, uint32_t nq, uint32_t k,
                             uint32_t nprobe, uint64_t *out_ids, float *out_d, uint32_t *out_cnt,
                             int32_t nthreads) {
  const int nt = nthreads_of(nthreads);
  const uint32_t d = s->d;
  DgoIndex qi{};  // quantizer view for quantized_distance / prepare
  qi.d = d;
  qi.metric = s->metric;
  qi.quant = s->quant;
  qi.code_size = s->code_size;
  qi.pq_M = s->pq_M;
  qi.pq_K = s->pq_K;
  qi.pq_codebooks = s->pq_codebooks;
  qi.int8_scale = s->int8_scale;
  qi.int8_offset = s->int8_offset;
  qi.rq_padded = s->rq_padded;
  qi.rq_signs = s->rq_signs;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
  for (int64_t t = 0; t < (int64_t)nq; ++t) {
    const float *q = Q + (uint64_t)t * d;
    std::vector<Cand> probes;
    for (uint32_t b = 0; b < s->num_blocks; ++b)
      if (s->block_live[b]) probes.push_back(Cand{metric_eval(s->metric, q, s->centroids + (uint64_t)b * d, d), b});
    std::sort(probes.begin(), probes.end(), lex_less);
    if (probes.size() > std::max(nprobe, 1u)) probes.resize(std::max(nprobe, 1u));
    std::vector<std::pair<uint64_t, float>> out;
    if (!probes.empty()) {
      const float d0 = probes[0].d;
      const float ratio = s->probe_ratio;
      size_t np = 0;
      while (np < probes.size() &&
             !(std::isfinite(ratio) && d0 >= 0.0f && probes[np].d > d0 * std::max(ratio, 1.0f)))
        ++np;
      probes.resize(np);
      auto entry_code = [&](uint32_t b, uint32_t i) {
        return s->entry_codes + ((uint64_t)b * s->block_cap + i) * s->code_size;
      };
      auto lt = [](const std::pair<float, uint64_t> &a, const std::pair<float, uint64_t> &b) {
        return a.first < b.first || (a.first == b.first && a.second < b.second);
      };
      std::priority_queue<std::pair<float, uint64_t>, std::vector<std::pair<float, uint64_t>>,
                          decltype(lt)>
          heap(lt);
      const bool l2 = s->metric == DGO_L2;
      if (s->quant == DGO_Q_RABITQ && (l2 || s->metric == DGO_L2SQ)) {
        // search_rabitq (:731-770): exact distance only when est - err < kth.
        std::vector<uint64_t> planes(4 * (s->rq_padded / 64));
        float k5[5];
        for (auto &pb : probes) {
          const uint32_t b = pb.id;
          rq_query(q, d, s->rq_padded, s->centroids + (uint64_t)b * d, s->rq_signs, planes.data(), k5);
          for (uint32_t i = 0; i < s->block_len[b]; ++i) {
            uint64_t id = s->entry_ids[(uint64_t)b * s->block_cap + i];
            if (s->deleted[id]) continue;
            float est, err;
            rq_est_bound(planes.data(), k5, entry_code(b, i), s->rq_padded, est, err);
            float kth = heap.size() < k ? kInf : heap.top().first;
            if (est - err < kth) {
              float ex = l2sq(q, s->raw + id * d, d);
              std::pair<float, uint64_t> c{ex, id};
              if (heap.size() < k) heap.push(c);
              else if (lt(c, heap.top())) {
                heap.pop();
                heap.push(c);
              }
            }
          }
        }
        while (!heap.empty()) {
          out.push_back({heap.top().second, l2 ? std::sqrt(heap.top().first) : heap.top().first});
          heap.pop();
        }
      } else {
        Prepared prep;
        if (s->quant != DGO_Q_NONE && s->quant != DGO_Q_RABITQ) prepare(qi, q, prep);
        const bool rerank = s->quant != DGO_Q_NONE && s->rerank_size > 0;
        const uint32_t want = rerank ? std::max(k, s->rerank_size) : k;
        std::vector<float> scratch;
        for (auto &pb : probes) {
          const uint32_t b = pb.id;
          for (uint32_t i = 0; i < s->block_len[b]; ++i) {
            uint64_t id = s->entry_ids[(uint64_t)b * s->block_cap + i];
            if (s->deleted[id]) continue;
            const uint8_t *code = entry_code(b, i);
            float dist;
            if (s->quant == DGO_Q_NONE) {
              dist = metric_eval(s->metric, q, (const float *)code, d);
            } else if (s->quant == DGO_Q_RABITQ) {  // non-L2 RaBitQ decodes (:346-349)
              scratch.resize(d);
              rq_decode(code, d, s->rq_padded, s->centroids + (uint64_t)b * d, s->rq_signs, scratch.data());
              dist = metric_eval(s->metric, q, scratch.data(), d);
            } else {
              DgoIndex one = qi;
              one.codes = code;
              dist = quantized_distance(one, q, 0, prep, scratch);
            }
            std::pair<float, uint64_t> c{dist, id};
            if (heap.size() < want) heap.push(c);
            else if (lt(c, heap.top())) {
              heap.pop();
              heap.push(c);
            }
          }
        }
        while (!heap.empty()) {
          out.push_back({heap.top().second, heap.top().first});
          heap.pop();
        }
        if (rerank)
          for (auto &r : out) r.second = metric_eval(s->metric, q, s->raw + r.first * d, d);
      }
      std::sort(out.begin(), out.end(), [](const std::pair<uint64_t, float> &a, const std::pair<uint64_t, float> &b) {
        return a.second < b.second || (a.second == b.second && a.first < b.first);
      });
      if (out.size() > k) out.resize(k);
    }
    for (uint32_t j = 0; j < k; ++j) {
      out_ids[(uint64_t)t * k + j] = j < out.size() ? out[j].first : UINT64_MAX;
      out_d[(uint64_t)t * k + j] = j < out.size() ? out[j].second : kInf;
    }
    out_cnt[t] = (uint32_t)std::min<size_t>(out.size(), k);
  }
  return 0;
}

void dgo_exact_knn(const float *X, uint64_t n, uint32_t d, const float *Q, uint32_t nq, uint32_t k,
                   int32_t metric, uint32_t *ids, double *dists, int32_t nthreads) {
  const int nt = nthreads_of(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (int64_t t = 0; t < (int64_t)nq; ++t) {
    const float *q = Q + (uint64_t)t * d;
    std::vector<std::pair<double, uint32_t>> all(n);
    for (uint64_t i = 0; i < n; ++i) {
      const float *x = X + i * d;
      double v;
      if (metric == DGO_L2SQ || metric == DGO_L2) {
        double s = 0.0;
        for (uint32_t j = 0; j < d; ++j) {
          double u = (double)q[j] - (double)x[j];
          s += u * u;
        }
        v = metric == DGO_L2 ? std::sqrt(s) : s;
      } else {
        double ab = 0.0, aa = 0.0, bb = 0.0;
        for (uint32_t j = 0; j < d; ++j) {
          ab += (double)q[j] * (double)x[j];
          aa += (double)q[j] * (double)q[j];
          bb += (double)x[j] * (double)x[j];
        }
        v = metric == DGO_COSINE ? ((aa == 0.0 || bb == 0.0) ? 1.0 : 1.0 - ab / (std::sqrt(aa) * std::sqrt(bb)))
                                 : 1.0 - ab;
      }
      all[i] = {v, (uint32_t)i};
    }
    uint32_t kk = (uint32_t)std::min<uint64_t>(k, n);
    std::partial_sort(all.begin(), all.begin() + kk, all.end());
    for (uint32_t j = 0; j < k; ++j) {
      ids[(uint64_t)t * k + j] = j < kk ? all[j].second : DGO_PAD;
      dists[(uint64_t)t * k + j] = j < kk ? all[j].first : std::numeric_limits<double>::infinity();
    }
  }
}

}  // extern "C"
