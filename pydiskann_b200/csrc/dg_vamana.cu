// dg_vamana.cu -- build_vamana_graph (diskann-rs src/lib.rs:774-1073) on the GPU.
//
// Each refinement pass of the reference reads a snapshot of the graph, so it
// is data parallel over nodes:
//   1. k_build_search: one warp per node runs the three greedy searches
//      (medoid + two random seeds, src/lib.rs:823-844) on the snapshot and
//      writes the node's candidate pool (current neighbours + the three
//      working sets) as (distance, id) keys;
//   2. k_prune: one block per node sorts and de-duplicates the pool and runs
//      robust_prune (src/lib.rs:977-1034) with the candidate rows staged in
//      shared memory;
//   3. symmetrisation (src/lib.rs:868-904): in-degree count, prefix sum,
//      incoming lists, distances, and k_prune again.
// The random draws use the counter-based stream shared with the oracle, so a
// GPU build equals the oracle build whenever distances are exact (integer
// valued data), which the tests check.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "dg_index.h"
#include "dg_search.cuh"

namespace dg {

constexpr int kPruneThreads = 256;
constexpr int kPruneSortCap = 2048;  // pools up to this size are sorted in shared memory
constexpr int kPruneTileBytes = 64 * 1024;

// --------------------------------------------------------------- bootstrap
// src/lib.rs:786-799: `target` distinct random neighbours != i, in draw order.
__global__ void k_bootstrap(uint64_t n, uint32_t R, uint32_t target, uint64_t seed, uint32_t *graph) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = gw; i < n; i += nw) {
    uint32_t *row = graph + i * R;
    uint32_t have = 0;
    for (uint64_t t0 = 0; have < target; t0 += 32) {
      const uint32_t x = (uint32_t)range_of(rand4(seed, 0, i, t0 + lane), n);
      bool ok = x != (uint32_t)i;
      // first occurrence within this batch of draws
      const uint32_t same = __match_any_sync(kFull, x);
      if (__ffs(same) - 1 != lane) ok = false;
      // not accepted by an earlier batch
      for (uint32_t j = 0; j < have && ok; ++j)
        if (row[j] == x) ok = false;
      const uint32_t m = __ballot_sync(kFull, ok);
      const uint32_t pos = have + __popc(m & ((1u << lane) - 1u));
      if (ok && pos < target) row[pos] = x;
      have = min(target, have + (uint32_t)__popc(m));
      __syncwarp();
    }
    for (uint32_t j = target + lane; j < R; j += 32) row[j] = DG_PAD;
  }
}

// -------------------------------------------------------- build searches
struct BuildArgs {
  uint64_t n;
  uint32_t d, dpad, R, Lb, medoid, pass;
  uint64_t seed;
  int32_t metric;
  const float *vf;      // [n][dpad]
  const uint16_t *vb;   // [n][dpad] bf16 (only when every value is bf16-exact)
  const uint32_t *graph;  // snapshot [n][R]
  uint32_t hbits, hB;     // visited table: log2 words, id bits
  uint64_t u0, u1;        // node range of this chunk
  uint32_t cw;            // candidate slots per node (R + 3*Lb)
  uint64_t *cand;         // [(u1-u0)][cw]
  uint32_t *cand_cnt;     // [(u1-u0)]
};

template <int ELEM, int MET, int LPR>
__device__ __forceinline__ float build_dist(const BuildArgs &a, const float *qs, uint32_t cand, int cnt,
                                            int lane) {
  if (ELEM == 1)
    return rows_distance<LPR, 1, MET>(reinterpret_cast<const uint8_t *>(a.vb), a.dpad * 2,
                                      (a.dpad / 8) / LPR, qs, cand, cnt, lane, a.metric == DG_L2, 0.0f);
  return rows_distance<LPR, 0, MET>(reinterpret_cast<const uint8_t *>(a.vf), a.dpad * 4,
                                    (a.dpad / 4) / LPR, qs, cand, cnt, lane, a.metric == DG_L2, 0.0f);
}

// Squared norm for the angular metric is recomputed per row inside
// rows_distance; the query norm is passed through qq.
template <int ELEM, int MET, int LPR, int LCAP>
__global__ void __launch_bounds__(128) k_build_search(BuildArgs a, WarpLayout Ly) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *wsm = smem + (size_t)warp * Ly.total;
  uint64_t *W[2] = {reinterpret_cast<uint64_t *>(wsm + Ly.w0), reinterpret_cast<uint64_t *>(wsm + Ly.w1)};
  uint64_t *cst = reinterpret_cast<uint64_t *>(wsm + Ly.cstage);
  uint32_t *stage = reinterpret_cast<uint32_t *>(wsm + Ly.stage);
  const Visited vt{reinterpret_cast<uint32_t *>(wsm + Ly.hash), a.hbits, a.hB};
  float *qs = reinterpret_cast<float *>(wsm + Ly.qf);
  const uint64_t gw = blockIdx.x * (uint64_t)(blockDim.x >> 5) + warp;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t u = a.u0 + gw; u < a.u1; u += nw) {
    uint64_t *out = a.cand + (u - a.u0) * a.cw;
    for (uint32_t i = lane; i < a.dpad; i += 32) qs[i] = a.vf[u * a.dpad + i];
    __syncwarp();
    float qq = 0.0f;
    if (MET == MET_COS) {
      for (uint32_t i = lane; i < a.dpad; i += 32) qq = fmaf(qs[i], qs[i], qq);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) qq += __shfl_xor_sync(kFull, qq, o);
    }
    uint32_t nout = 0;
    // current neighbours with their distances (src/lib.rs:818-822)
    {
      const uint32_t *row = a.graph + u * a.R;
      for (uint32_t j0 = 0; j0 < a.R; j0 += 32) {
        const uint32_t j = j0 + lane;
        const uint32_t nb = j < a.R ? row[j] : DG_PAD;
        const bool ok = nb != DG_PAD;
        const uint32_t m = __ballot_sync(kFull, ok);
        const int cnt = __popc(m);
        if (!cnt) continue;
        if (ok) stage[__popc(m & ((1u << lane) - 1u))] = nb;
        __syncwarp();
        const uint32_t c = lane < cnt ? stage[lane] : 0u;
        float dd = rows_distance<LPR, ELEM == 1 ? 1 : 0, MET>(
            ELEM == 1 ? reinterpret_cast<const uint8_t *>(a.vb) : reinterpret_cast<const uint8_t *>(a.vf),
            ELEM == 1 ? a.dpad * 2 : a.dpad * 4, ELEM == 1 ? (a.dpad / 8) / LPR : (a.dpad / 4) / LPR, qs,
            c, cnt, lane, a.metric == DG_L2, qq);
        if (lane < cnt) out[nout + lane] = make_key(dd, c);
        nout += cnt;
        __syncwarp();
      }
    }
    // three greedy searches (greedy_search, src/lib.rs:921-973)
    const uint32_t seeds[3] = {a.medoid, (uint32_t)range_of(rand4(a.seed, a.pass + 1, u, 0), a.n),
                               (uint32_t)range_of(rand4(a.seed, a.pass + 1, u, 1), a.n)};
    for (int s = 0; s < 3; ++s) {
      vt.clear(lane);
      __syncwarp();
      int cur = 0, wsize = 1;
      {
        const uint32_t c = seeds[s];
        float dd = rows_distance<LPR, ELEM == 1 ? 1 : 0, MET>(
            ELEM == 1 ? reinterpret_cast<const uint8_t *>(a.vb) : reinterpret_cast<const uint8_t *>(a.vf),
            ELEM == 1 ? a.dpad * 2 : a.dpad * 4, ELEM == 1 ? (a.dpad / 8) / LPR : (a.dpad / 4) / LPR, qs,
            c, 1, lane, a.metric == DG_L2, qq);
        dd = __shfl_sync(kFull, dd, 0);
        if (lane == 0) {
          W[0][0] = make_key(dd, c);
          vt.test_and_set(c);
        }
        __syncwarp();
      }
      while (true) {
        int idx = -1;
        for (int base = 0; base < wsize; base += 32) {
          const int i = base + lane;
          const bool un = i < wsize && !key_expanded(W[cur][i]);
          const uint32_t m = __ballot_sync(kFull, un);
          if (m) {
            idx = base + __ffs(m) - 1;
            break;
          }
        }
        if (idx < 0) break;
        const uint64_t best = W[cur][idx];
        if (wsize >= (int)a.Lb && key_dist(best) >= key_dist(W[cur][a.Lb - 1])) break;
        if (lane == 0) W[cur][idx] = best | 1ull;
        const uint32_t *row = a.graph + (size_t)key_id(best) * a.R;
        int ns = 0;
        for (uint32_t j0 = 0; j0 < a.R; j0 += 32) {
          const uint32_t j = j0 + lane;
          const uint32_t nb = j < a.R ? __ldg(row + j) : DG_PAD;
          bool ok = nb != DG_PAD && nb < a.n;
          if (ok) ok = !vt.test_and_set(nb);
          const uint32_t m = __ballot_sync(kFull, ok);
          if (ok) stage[ns + __popc(m & ((1u << lane) - 1u))] = nb;
          ns += __popc(m);
        }
        __syncwarp();
        for (int g0 = 0; g0 < ns; g0 += 32) {
          const int cnt = min(32, ns - g0);
          const uint32_t c = lane < cnt ? stage[g0 + lane] : DG_PAD;
          const float dd = rows_distance<LPR, ELEM == 1 ? 1 : 0, MET>(
              ELEM == 1 ? reinterpret_cast<const uint8_t *>(a.vb) : reinterpret_cast<const uint8_t *>(a.vf),
              ELEM == 1 ? a.dpad * 2 : a.dpad * 4, ELEM == 1 ? (a.dpad / 8) / LPR : (a.dpad / 4) / LPR,
              qs, c, cnt, lane, a.metric == DG_L2, qq);
          const uint64_t key = lane < cnt ? make_key(dd, c) : kKeyInvalid;
          insert_batch(key, W, cur, wsize, (int)a.Lb, cst, lane);
        }
      }
      for (int i = lane; i < wsize; i += 32) out[nout + i] = strip_flag(W[cur][i]);
      nout += wsize;
      __syncwarp();
    }
    if (lane == 0) a.cand_cnt[u - a.u0] = nout;
    __syncwarp();
  }
}

// ------------------------------------------------------------------- prune
struct PruneArgs {
  uint64_t u0, nodes;
  const uint64_t *keys;     // candidate keys
  const uint64_t *off;      // per-node offset into keys (nodes entries) or null (fixed stride)
  uint64_t stride;          // fixed stride when off is null
  const uint32_t *cnt;      // per-node count
  uint64_t *gsort;          // global sort scratch for oversized pools: [gridDim][gcap]
  uint32_t gcap;
  const float *vf;
  const uint16_t *vb;
  uint32_t d, dpad, R;
  float alpha;
  int32_t metric;
  uint32_t tile_rows;
  uint32_t *out;            // [n][R]
};

// Distance between candidate rows j and i (rows staged in `tile` when < tile_rows).
template <int ELEM, int MET>
__device__ __forceinline__ float pair_dist(const PruneArgs &a, const uint32_t *tile, uint32_t tw,
                                           uint32_t j, uint32_t idj, uint32_t i, uint32_t idi) {
  float ab = 0.0f, aa = 0.0f, bb = 0.0f;
  const uint32_t words = ELEM == 1 ? a.dpad / 2 : a.dpad;
  const uint32_t *rj = j < a.tile_rows ? tile + (size_t)j * tw
                                       : (ELEM == 1 ? reinterpret_cast<const uint32_t *>(a.vb + (size_t)idj * a.dpad)
                                                    : reinterpret_cast<const uint32_t *>(a.vf + (size_t)idj * a.dpad));
  const uint32_t *ri = i < a.tile_rows ? tile + (size_t)i * tw
                                       : (ELEM == 1 ? reinterpret_cast<const uint32_t *>(a.vb + (size_t)idi * a.dpad)
                                                    : reinterpret_cast<const uint32_t *>(a.vf + (size_t)idi * a.dpad));
  for (uint32_t t = 0; t < words; ++t) {
    const uint32_t wj = rj[t], wi = ri[t];
    if (ELEM == 1) {
      const float xj0 = __uint_as_float(wj << 16), xj1 = __uint_as_float(wj & 0xffff0000u);
      const float xi0 = __uint_as_float(wi << 16), xi1 = __uint_as_float(wi & 0xffff0000u);
      if (MET == MET_L2) {
        const float t0 = xj0 - xi0, t1 = xj1 - xi1;
        ab = fmaf(t0, t0, ab);
        ab = fmaf(t1, t1, ab);
      } else {
        ab = fmaf(xj0, xi0, ab);
        ab = fmaf(xj1, xi1, ab);
        if (MET == MET_COS) {
          aa = fmaf(xj0, xj0, aa); aa = fmaf(xj1, xj1, aa);
          bb = fmaf(xi0, xi0, bb); bb = fmaf(xi1, xi1, bb);
        }
      }
    } else {
      const float xj = __uint_as_float(wj), xi = __uint_as_float(wi);
      if (MET == MET_L2) {
        const float t0 = xj - xi;
        ab = fmaf(t0, t0, ab);
      } else {
        ab = fmaf(xj, xi, ab);
        if (MET == MET_COS) {
          aa = fmaf(xj, xj, aa);
          bb = fmaf(xi, xi, bb);
        }
      }
    }
  }
  // metric_eval(X[j], X[i]) of the reference's prune_neighbors
  return finish_metric(MET, a.metric == DG_L2, ab, aa, bb);
}

template <int ELEM, int MET>
__global__ void __launch_bounds__(kPruneThreads) k_prune(PruneArgs a) {
  extern __shared__ __align__(16) uint8_t smem[];
  uint64_t *skeys = reinterpret_cast<uint64_t *>(smem);               // kPruneSortCap
  float *occ = reinterpret_cast<float *>(skeys + kPruneSortCap);        // kPruneSortCap
  uint8_t *sel = reinterpret_cast<uint8_t *>(occ + kPruneSortCap);      // kPruneSortCap
  uint32_t *tile = reinterpret_cast<uint32_t *>(sel + kPruneSortCap);
  __shared__ uint32_t s_m, s_np;
  __shared__ uint32_t s_out[kStageCap];
  const int tid = threadIdx.x;
  const uint32_t words = ELEM == 1 ? a.dpad / 2 : a.dpad;
  const uint32_t tw = words + 1;  // odd stride: rows land in distinct banks
  for (uint64_t b = blockIdx.x; b < a.nodes; b += gridDim.x) {
    const uint64_t u = a.u0 + b;
    const uint64_t off = a.off ? a.off[b] : b * a.stride;
    const uint32_t c = a.cnt[b];
    const uint64_t *src = a.keys + off;
    // sort the pool (self removed) in shared memory, or in global scratch when large
    uint32_t p2 = 1;
    while (p2 < c) p2 <<= 1;
    uint64_t *K = p2 <= (uint32_t)kPruneSortCap ? skeys : a.gsort + (size_t)blockIdx.x * a.gcap;
    for (uint32_t i = tid; i < p2; i += blockDim.x) {
      uint64_t k = i < c ? strip_flag(src[i]) : kKeyInvalid;
      if (k != kKeyInvalid && key_id(k) == (uint32_t)u) k = kKeyInvalid;
      K[i] = k;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= p2; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = tid; i < p2; i += blockDim.x) {
          const uint32_t l = i ^ j;
          if (l > i) {
            const uint64_t x = K[i], y = K[l];
            const bool up = (i & k) == 0;
            if ((x > y) == up) {
              K[i] = y;
              K[l] = x;
            }
          }
        }
        __syncthreads();
      }
    }
    // de-duplicate (same id => same key) and compact, keeping order
    if (tid == 0) {
      uint32_t m = 0;
      uint64_t prev = kKeyInvalid;
      for (uint32_t i = 0; i < p2; ++i) {
        const uint64_t k = K[i];
        if (k == kKeyInvalid) break;
        if (k == prev) continue;
        prev = k;
        K[m++] = k;
      }
      s_m = m;
      s_np = 0;
    }
    __syncthreads();
    const uint32_t m = s_m;
    // per-candidate state lives in shared memory for the first kPruneSortCap
    // candidates; larger pools keep it next to their keys in global scratch
    float *O = m <= (uint32_t)kPruneSortCap ? occ : reinterpret_cast<float *>(a.gsort + (size_t)blockIdx.x * a.gcap + a.gcap / 2);
    uint8_t *S = m <= (uint32_t)kPruneSortCap ? sel : reinterpret_cast<uint8_t *>(O + a.gcap / 2);
    for (uint32_t i = tid; i < m; i += blockDim.x) {
      O[i] = 0.0f;
      S[i] = 0;
    }
    // stage candidate rows
    const uint32_t rows = min(m, a.tile_rows);
    for (uint32_t e = tid; e < rows * words; e += blockDim.x) {
      const uint32_t r = e / words, t = e % words;
      const uint32_t id = key_id(K[r]);
      tile[(size_t)r * tw + t] = ELEM == 1 ? reinterpret_cast<const uint32_t *>(a.vb + (size_t)id * a.dpad)[t]
                                           : __float_as_uint(a.vf[(size_t)id * a.dpad + t]);
    }
    __syncthreads();
    // robust_prune (src/lib.rs:977-1034)
    const float alpha = fmaxf(a.alpha, 1.0f);
    float cur_alpha = 1.0f;
    uint32_t np = 0;
    // Every thread takes the same decisions from S/O: the flag of the entry
    // being decided is written only after the barrier that ends its selection,
    // and each pass ends with a barrier, so no thread can read a flag in the
    // middle of its update and skip a barrier the others wait at.
    while (cur_alpha <= alpha && np < a.R) {
      for (uint32_t i = 0; i < m; ++i) {
        if (np >= a.R) break;
        if (S[i] || O[i] > cur_alpha) continue;
        const uint32_t idi = key_id(K[i]);
        if (tid == 0) s_out[np] = idi;
        ++np;
        for (uint32_t j = i + 1 + tid; j < m; j += blockDim.x) {
          if (S[j] || O[j] > alpha) continue;
          const uint64_t kj = K[j];
          const float djk = pair_dist<ELEM, MET>(a, tile, tw, j, key_id(kj), i, idi);
          O[j] = djk == 0.0f ? __int_as_float(0x7f800000) : fmaxf(O[j], __fdiv_rn(key_dist(kj), djk));
        }
        __syncthreads();
        if (tid == 0) S[i] = 1;
      }
      __syncthreads();
      cur_alpha = __fmul_rn(cur_alpha, 1.2f);
    }
    if (tid == 0) {
      for (uint32_t i = 0; i < m && np < a.R; ++i)
        if (!S[i]) {
          S[i] = 1;
          s_out[np++] = key_id(K[i]);
        }
      s_np = np;
    }
    __syncthreads();
    uint32_t *row = a.out + u * a.R;
    for (uint32_t j = tid; j < a.R; j += blockDim.x) row[j] = j < s_np ? s_out[j] : DG_PAD;
    __syncthreads();
  }
}

// ---------------------------------------------------------- symmetrisation
__global__ void k_degrees(const uint32_t *g, uint64_t n, uint32_t R, uint32_t *outdeg, uint32_t *indeg) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n * R;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = g[e];
    if (v != DG_PAD) {
      atomicAdd(indeg + v, 1u);
      atomicAdd(outdeg + e / R, 1u);
    }
  }
}
__global__ void k_pool_sizes(const uint32_t *outdeg, const uint32_t *indeg, uint64_t n, uint64_t *sz) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    sz[i] = (uint64_t)outdeg[i] + indeg[i];
}
// pool ids of node u: its outgoing list, then everyone pointing at u
__global__ void k_fill_pools(const uint32_t *g, uint64_t n, uint32_t R, const uint64_t *off,
                             const uint32_t *outdeg, uint32_t *cursor, uint32_t *pool_ids) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n * R;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = g[e];
    if (v == DG_PAD) continue;
    const uint64_t u = e / R;
    pool_ids[off[u] + (e % R)] = v;  // outgoing lists are packed at the row front
    const uint32_t pos = atomicAdd(cursor + v, 1u);
    pool_ids[off[v] + outdeg[v] + pos] = (uint32_t)u;
  }
}
// distances of every pool entry to its node (warp per node)
template <int ELEM, int MET, int LPR>
__global__ void k_pool_keys(const float *vf, const uint16_t *vb, uint64_t n, uint32_t dpad, int metric,
                            const uint64_t *off, const uint32_t *pool_ids, uint64_t *keys, uint32_t *cnt) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  extern __shared__ __align__(16) float qsm[];
  float *qs = qsm + (size_t)warp * dpad;
  const uint64_t gw = blockIdx.x * (uint64_t)(blockDim.x >> 5) + warp;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t u = gw; u < n; u += nw) {
    for (uint32_t i = lane; i < dpad; i += 32) qs[i] = vf[u * dpad + i];
    __syncwarp();
    float qq = 0.0f;
    if (MET == MET_COS) {
      for (uint32_t i = lane; i < dpad; i += 32) qq = fmaf(qs[i], qs[i], qq);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) qq += __shfl_xor_sync(kFull, qq, o);
    }
    const uint64_t b = off[u], e = off[u + 1];
    for (uint64_t g0 = b; g0 < e; g0 += 32) {
      const int c = (int)((e - g0) < 32 ? (e - g0) : 32);
      const uint32_t id = lane < c ? pool_ids[g0 + lane] : 0u;
      const float dd = rows_distance<LPR, ELEM == 1 ? 1 : 0, MET>(
          ELEM == 1 ? reinterpret_cast<const uint8_t *>(vb) : reinterpret_cast<const uint8_t *>(vf),
          ELEM == 1 ? dpad * 2 : dpad * 4, ELEM == 1 ? (dpad / 8) / LPR : (dpad / 4) / LPR, qs, id, c, lane,
          metric == DG_L2, qq);
      if (lane < c) keys[g0 + lane] = make_key(dd, id);
    }
    if (lane == 0) cnt[u] = (uint32_t)(e - b);
    __syncwarp();
  }
}

__global__ void k_bf16_exact(const float *v, uint64_t total, unsigned int *flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float x = v[i];
    if (__uint_as_float(__float_as_uint(x) & 0xffff0000u) != x) atomicOr(flag, 1u);
  }
}

static uint32_t id_bits(uint64_t n) {
  uint32_t b = 1;
  while (b < 32 && (1ull << b) < n) ++b;
  return b;
}

template <int ELEM, int MET>
static DgStatus run_build(const BuildArgs &base, float *vf, uint16_t *vb, uint32_t *g0, uint32_t *g1,
                          float alpha, cudaStream_t st, uint32_t **result) {
  const uint64_t n = base.n;
  const uint32_t R = base.R, dpad = base.dpad;
  constexpr int LPR = ELEM == 1 ? 4 : 8;
  const int lcap = base.Lb <= 64 ? 64 : base.Lb <= 256 ? 256 : 1024;
  int dev = 0, sms = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // candidate pools of the search phase, processed in node chunks
  const uint32_t cw = R + 3 * base.Lb;
  const uint64_t chunk = std::min<uint64_t>(n, 1ull << 18);
  uint64_t *cand = nullptr;
  uint32_t *ccnt = nullptr;
  DG_CUDA(cudaMallocAsync(&cand, chunk * cw * 8, st));
  DG_CUDA(cudaMallocAsync(&ccnt, chunk * 4, st));
  // prune geometry
  const uint32_t words = ELEM == 1 ? dpad / 2 : dpad;
  uint32_t tile_rows = (uint32_t)(kPruneTileBytes / ((words + 1) * 4));
  if (tile_rows < 1) tile_rows = 1;
  const size_t psmem = (size_t)kPruneSortCap * (8 + 4 + 1) + (size_t)tile_rows * (words + 1) * 4;
  auto prune_k = k_prune<ELEM, MET>;
  DG_CUDA(cudaFuncSetAttribute(prune_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem));
  int pblocks = 0;
  DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pblocks, prune_k, kPruneThreads, psmem));
  const int pgrid = std::max(1, pblocks) * sms;
  // search kernel geometry
  const uint32_t hbits = base.Lb <= 64 ? 10 : base.Lb <= 128 ? 11 : 12;
  const WarpLayout Ly = warp_layout(ELEM == 1 ? TRAV_BF16 : TRAV_F32, lcap, false, hbits, dpad, 0, 0, 0);
  void (*sk)(BuildArgs, WarpLayout) = lcap == 64 ? k_build_search<ELEM, MET, LPR, 64>
                                    : lcap == 256 ? k_build_search<ELEM, MET, LPR, 256>
                                                  : k_build_search<ELEM, MET, LPR, 1024>;
  DG_CUDA(cudaFuncSetAttribute(sk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(Ly.total * 4)));
  int sblocks = 0;
  DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sblocks, sk, 128, Ly.total * 4));
  if (sblocks < 1) return fail(DG_ENOTSUP, "build search state does not fit in shared memory");
  // symmetrisation buffers
  uint32_t *outdeg = nullptr, *indeg = nullptr, *cursor = nullptr, *pool_ids = nullptr, *pcnt = nullptr;
  uint64_t *psz = nullptr, *poff = nullptr, *pkeys = nullptr;
  DG_CUDA(cudaMallocAsync(&outdeg, n * 4, st));
  DG_CUDA(cudaMallocAsync(&indeg, n * 4, st));
  DG_CUDA(cudaMallocAsync(&cursor, n * 4, st));
  DG_CUDA(cudaMallocAsync(&pcnt, n * 4, st));
  DG_CUDA(cudaMallocAsync(&psz, (n + 1) * 8, st));
  DG_CUDA(cudaMallocAsync(&poff, (n + 1) * 8, st));
  DG_CUDA(cudaMallocAsync(&pool_ids, n * R * 2 * 4, st));
  DG_CUDA(cudaMallocAsync(&pkeys, n * R * 2 * 8, st));
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, psz, poff, n + 1, st);
  void *scan_tmp = nullptr;
  DG_CUDA(cudaMallocAsync(&scan_tmp, scan_bytes, st));
  // global sort scratch for pools above the shared-memory capacity
  const uint32_t gcap = (uint32_t)std::max<uint64_t>(4096, 2 * (uint64_t)(cw + 2 * R));
  uint64_t *gsort = nullptr;
  // sized generously: pools larger than this are clipped by a pre-check below
  uint32_t gcap_sym = gcap;
  uint32_t *cur = g0, *nxt = g1;
  for (uint32_t pass = 0; pass < 2; ++pass) {
    BuildArgs a = base;
    a.pass = pass;
    a.graph = cur;
    a.hbits = hbits;
    a.hB = std::max(id_bits(n), hbits);
    a.cw = cw;
    a.cand = cand;
    a.cand_cnt = ccnt;
    for (uint64_t u0 = 0; u0 < n; u0 += chunk) {
      a.u0 = u0;
      a.u1 = std::min(n, u0 + chunk);
      const uint64_t nodes = a.u1 - a.u0;
      const int grid = (int)std::min<uint64_t>((uint64_t)sblocks * sms, (nodes + 3) / 4);
      sk<<<grid, 128, Ly.total * 4, st>>>(a, Ly);
      DG_CUDA(cudaGetLastError());
      PruneArgs p{};
      p.u0 = u0;
      p.nodes = nodes;
      p.keys = cand;
      p.off = nullptr;
      p.stride = cw;
      p.cnt = ccnt;
      p.vf = vf;
      p.vb = vb;
      p.d = base.d;
      p.dpad = dpad;
      p.R = R;
      p.alpha = alpha;
      p.metric = base.metric;
      p.tile_rows = tile_rows;
      p.out = nxt;
      if (cw > (uint32_t)kPruneSortCap) {
        if (!gsort) DG_CUDA(cudaMallocAsync(&gsort, (size_t)pgrid * gcap * 8, st));
        p.gsort = gsort;
        p.gcap = gcap;
      }
      k_prune<ELEM, MET><<<(int)std::min<uint64_t>(pgrid, nodes), kPruneThreads, psmem, st>>>(p);
      DG_CUDA(cudaGetLastError());
    }
    // symmetrise: union of outgoing and incoming, distances, prune into `cur`
    DG_CUDA(cudaMemsetAsync(outdeg, 0, n * 4, st));
    DG_CUDA(cudaMemsetAsync(indeg, 0, n * 4, st));
    DG_CUDA(cudaMemsetAsync(cursor, 0, n * 4, st));
    DG_CUDA(cudaMemsetAsync(psz, 0, (n + 1) * 8, st));
    k_degrees<<<sms * 8, 256, 0, st>>>(nxt, n, R, outdeg, indeg);
    k_pool_sizes<<<sms * 8, 256, 0, st>>>(outdeg, indeg, n, psz);
    cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, psz, poff, n + 1, st);
    k_fill_pools<<<sms * 8, 256, 0, st>>>(nxt, n, R, poff, outdeg, cursor, pool_ids);
    const int kw = 4;
    k_pool_keys<ELEM, MET, LPR><<<sms * 16, kw * 32, kw * dpad * 4, st>>>(vf, vb, n, dpad, base.metric, poff,
                                                                         pool_ids, pkeys, pcnt);
    DG_CUDA(cudaGetLastError());
    // the largest pool decides whether global sort scratch is needed
    uint32_t max_in = 0;
    {
      std::vector<uint32_t> hin(n);
      DG_CUDA(cudaMemcpyAsync(hin.data(), indeg, n * 4, cudaMemcpyDeviceToHost, st));
      DG_CUDA(cudaStreamSynchronize(st));
      for (uint32_t v : hin) max_in = std::max(max_in, v);
    }
    uint64_t maxpool = (uint64_t)R + max_in;
    PruneArgs p{};
    p.u0 = 0;
    p.nodes = n;
    p.keys = pkeys;
    p.off = poff;
    p.cnt = pcnt;
    p.vf = vf;
    p.vb = vb;
    p.d = base.d;
    p.dpad = dpad;
    p.R = R;
    p.alpha = alpha;
    p.metric = base.metric;
    p.tile_rows = tile_rows;
    p.out = cur;
    if (maxpool > (uint64_t)kPruneSortCap) {
      uint32_t need = 1;
      while (need < maxpool) need <<= 1;
      need = std::max<uint32_t>(need * 2, 4096);  // keys, then occlusion + flags
      if (need > gcap_sym || !gsort) {
        if (gsort) DG_CUDA(cudaFreeAsync(gsort, st));
        gcap_sym = need;
        DG_CUDA(cudaMallocAsync(&gsort, (size_t)pgrid * gcap_sym * 8, st));
      }
      p.gsort = gsort;
      p.gcap = gcap_sym;
    }
    k_prune<ELEM, MET><<<(int)std::min<uint64_t>(pgrid, n), kPruneThreads, psmem, st>>>(p);
    DG_CUDA(cudaGetLastError());
  }
  DG_CUDA(cudaStreamSynchronize(st));
  cudaFreeAsync(cand, st);
  cudaFreeAsync(ccnt, st);
  cudaFreeAsync(outdeg, st);
  cudaFreeAsync(indeg, st);
  cudaFreeAsync(cursor, st);
  cudaFreeAsync(pcnt, st);
  cudaFreeAsync(psz, st);
  cudaFreeAsync(poff, st);
  cudaFreeAsync(pool_ids, st);
  cudaFreeAsync(pkeys, st);
  cudaFreeAsync(scan_tmp, st);
  if (gsort) cudaFreeAsync(gsort, st);
  *result = cur;
  return DG_OK;
}

}  // namespace dg

using namespace dg;

extern "C" DgStatus dg_build_vamana(const float *X, uint64_t n, uint32_t dim, int32_t metric, uint32_t R,
                                    uint32_t build_beam, float alpha, uint64_t seed, uint32_t medoid,
                                    int32_t device, uint32_t *out_adjacency) {
  if (!X || !out_adjacency || n == 0 || dim == 0) return fail(DG_EINVAL, "bad build arguments");
  if (n >= (1ull << 31)) return fail(DG_EINVAL, "num_vectors must be < 2^31");
  if (R == 0 || R > (uint32_t)kStageCap) return fail(DG_EINVAL, "max_degree must be in [1, 256]");
  if (build_beam == 0 || build_beam > 1024) return fail(DG_EINVAL, "build_beam_width must be in [1, 1024]");
  if (medoid >= n) return fail(DG_EINVAL, "medoid out of range");
  if (metric < DG_L2SQ || metric > DG_DOT) return fail(DG_EINVAL, "unknown metric");
  DG_CUDA(cudaSetDevice(device));
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const uint32_t dpad = dpad_of(dim);
  float *vf = nullptr;
  uint16_t *vb = nullptr;
  uint32_t *g0 = nullptr, *g1 = nullptr;
  unsigned int *flag = nullptr;
  DgStatus s = DG_OK;
  if (cudaMallocAsync(&vf, n * dpad * 4, st) != cudaSuccess || cudaMallocAsync(&g0, n * R * 4, st) != cudaSuccess ||
      cudaMallocAsync(&g1, n * R * 4, st) != cudaSuccess || cudaMallocAsync(&flag, 4, st) != cudaSuccess)
    s = fail(DG_ENOMEM, "build staging");
  if (s == DG_OK) s = upload_rows_f32(X, n, dim, dpad, vf, st);
  bool exact_bf16 = false;
  if (s == DG_OK) {
    // BF16 rows carry the same values when every coordinate is bf16-exact
    // (integer data in [-256, 256], BF16-stored embeddings): half the gather bytes.
    cudaMemsetAsync(flag, 0, 4, st);
    k_bf16_exact<<<148 * 8, 256, 0, st>>>(vf, n * dpad, flag);
    unsigned int hf = 1;
    cudaMemcpyAsync(&hf, flag, 4, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    exact_bf16 = hf == 0 && metric != DG_COSINE;
    if (exact_bf16) {
      if (cudaMallocAsync(&vb, n * dpad * 2, st) != cudaSuccess) s = fail(DG_ENOMEM, "build staging");
      else s = encode_bf16_device(vf, n, dpad, vb, st);
    }
  }
  if (s == DG_OK) {
    const uint32_t target = (uint32_t)std::min<uint64_t>(std::max<uint32_t>(R / 2, 2u), n - 1);
    k_bootstrap<<<148 * 8, 256, 0, st>>>(n, R, target, seed, g0);
    if (cudaGetLastError() != cudaSuccess) s = fail(DG_EDEVICE, "bootstrap launch");
  }
  uint32_t *result = nullptr;
  if (s == DG_OK) {
    BuildArgs a{};
    a.n = n;
    a.d = dim;
    a.dpad = dpad;
    a.R = R;
    a.Lb = build_beam;
    a.medoid = medoid;
    a.seed = seed;
    a.metric = metric;
    a.vf = vf;
    a.vb = vb;
    const int met = metric == DG_DOT ? MET_DOT : metric == DG_COSINE ? MET_COS : MET_L2;
    if (exact_bf16) {
      s = met == MET_DOT ? run_build<1, MET_DOT>(a, vf, vb, g0, g1, alpha, st, &result)
                         : run_build<1, MET_L2>(a, vf, vb, g0, g1, alpha, st, &result);
    } else {
      s = met == MET_DOT   ? run_build<0, MET_DOT>(a, vf, vb, g0, g1, alpha, st, &result)
          : met == MET_COS ? run_build<0, MET_COS>(a, vf, vb, g0, g1, alpha, st, &result)
                           : run_build<0, MET_L2>(a, vf, vb, g0, g1, alpha, st, &result);
    }
  }
  if (s == DG_OK) {
    if (cudaMemcpyAsync(out_adjacency, result, n * R * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      s = fail(DG_EDEVICE, std::string("build failed: ") + cudaGetErrorString(cudaGetLastError()));
  }
  if (vf) cudaFreeAsync(vf, st);
  if (vb) cudaFreeAsync(vb, st);
  if (g0) cudaFreeAsync(g0, st);
  if (g1) cudaFreeAsync(g1, st);
  if (flag) cudaFreeAsync(flag, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}
