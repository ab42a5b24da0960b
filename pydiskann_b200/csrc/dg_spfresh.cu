// dg_spfresh.cu -- SPFresh posting-list search on the GPU (diskann-rs
// src/spfresh.rs:344-378, 671-770).
//
// One warp per query, persistent grid with a work counter:
//   1. routing: the distance from the query to every live posting centroid,
//      each summed sequentially in the order the oracle sums it (by one lane
//      in this kernel for few postings, by the tiled k_route for >= 512),
//      kept as the nprobe smallest (distance, posting) keys (nearest,
//      src/spfresh.rs:358-378; brute force at every posting count);
//   2. the probe_ratio cut (:683-687);
//   3. the scan of every probed posting: tombstoned ids skipped, the
//      distance of each entry's code (raw f32, PQ, int8, F16) inserted into
//      the `want` smallest (distance, id) keys (:702-717), then the exact FP32
//      rerank from the raw store (:719-723);
//   4. RaBitQ codes with an L2 metric follow search_rabitq (:731-770): a
//      per-posting residual query, and an exact distance only for entries whose
//      lower bound est - err beats the current k-th exact distance.  The
//      threshold changes after every insertion, so the warp computes a batch of
//      candidates in parallel and replays the decisions entry by entry.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "dg_index.h"
#include "dg_search.cuh"

struct DgSpfresh {
  int device = 0;
  uint32_t d = 0, dpad = 0, nblocks = 0, cap = 0;
  int32_t metric = DG_L2SQ;
  int32_t quant = DG_Q_NONE;
  uint32_t code_size = 0, code_stride = 0;
  float *centroids = nullptr;  // [nblocks][dpad]
  uint8_t *live = nullptr;     // [nblocks]
  uint32_t *len = nullptr;     // [nblocks]
  uint32_t *ids = nullptr;     // [nblocks][cap]
  uint8_t *codes = nullptr;    // [nblocks][cap][code_stride]
  uint64_t id_cap = 0;
  uint32_t *deleted = nullptr; // bitmap over ids
  float *raw = nullptr;        // [id_cap][dpad]
  uint32_t pq_M = 0, pq_K = 0;
  float *pq_cb = nullptr;
  float i8_scale = 1.0f, i8_offset = 0.0f;
  uint32_t rq_padded = 0;
  float *rq_signs = nullptr;
  uint32_t *counter = nullptr;
  cudaStream_t stream = nullptr;
  // recorded after each search on its stream: the next search (which reuses
  // the same scratch) and every update wait for it on the GPU, so a search
  // issued on a caller's stream never has its scratch or postings rewritten
  // under it
  cudaEvent_t searched = nullptr;
  std::mutex mu;
  std::vector<void *> allocs;
  DgIndex::Buf q, oids, od, ocnt, route;  // route: query x posting routing distances of one chunk
  DgIndex::Buf live_idx;                   // [0]: number of live postings, then their slot indices
  DgIndex::Buf fr;                         // tensor-core routing: centre, norms and scales, FP16 halves
  // posting-major scan of one chunk: probes per query, (query, posting) pairs
  // grouped by posting, work items, per-pair candidate lists
  DgIndex::Buf probe, probe_cnt, pcount, pstart, pfill, istart, pair_q, pos_of, items, pair_keys, pair_cnt, misc;
  DgIndex::Buf qthr;  // posting-major scan: per query, a bound of its k-th distance
};

namespace dg {

struct SpfArgs {
  uint32_t d, dpad, nblocks, cap;
  int32_t metric;
  const float *centroids;
  const uint8_t *live;
  const uint32_t *len;
  const uint32_t *ids;
  const uint8_t *codes;
  uint32_t code_stride;
  const uint32_t *deleted;
  const float *raw;
  uint32_t pq_M, pq_K, pq_ds;
  const float *pq_cb;
  float i8_scale, i8_offset;
  uint32_t rq_padded;
  const float *rq_signs;
  const float *Q;
  uint32_t nq, k, nprobe, rerank;
  float probe_ratio;
  uint64_t *out_ids;
  float *out_d;
  uint32_t *out_cnt;
  uint32_t *counter;
  const float *route;        // [nq][nblocks] routing distances (null: computed in the scan kernel)
  const uint32_t *route_idx; // [1 + live] count, then the live slots the columns of `route` belong to
  uint32_t *probe_out;       // non-null: write each query's probed slots ([nq][nprobe]) and stop
  uint32_t *probe_cnt;       // [nq] number of probed slots
  const uint32_t *probe_in;  // non-null: each query's probed slots ([nq][nprobe], ascending keys), routing done
  const uint32_t *probe_in_cnt;
};

enum SpfKind { SPF_RAW = 0, SPF_PQ = 1, SPF_INT8 = 2, SPF_F16 = 3, SPF_RABITQ = 4 };

// The float whose ordered bits (ordered_bits) are u.
__device__ __forceinline__ float ordered_float(uint32_t u) {
  u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  return __uint_as_float(u);
}

// metric_eval of the oracle with its rounding (sequential sums).
__device__ __forceinline__ float seq_metric(const float *q, const float *x, uint32_t d, int metric) {
  if (metric == DG_L2SQ || metric == DG_L2) {
    float acc = 0.0f;
    for (uint32_t i = 0; i < d; ++i) {
      const float t = __fsub_rn(q[i], __ldg(x + i));
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
    return metric == DG_L2 ? __fsqrt_rn(acc) : acc;
  }
  float ab = 0.0f, aa = 0.0f, bb = 0.0f;
  for (uint32_t i = 0; i < d; ++i) {
    const float xv = __ldg(x + i);
    ab = __fadd_rn(ab, __fmul_rn(q[i], xv));
    aa = __fadd_rn(aa, __fmul_rn(q[i], q[i]));
    bb = __fadd_rn(bb, __fmul_rn(xv, xv));
  }
  if (metric == DG_DOT) return __fsub_rn(1.0f, ab);
  if (aa == 0.0f && bb == 0.0f) return 0.0f;
  if (ab == 0.0f) return 1.0f;
  const float r = __fsub_rn(1.0f, __fdiv_rn(ab, __fmul_rn(__fsqrt_rn(aa), __fsqrt_rn(bb))));
  return r > 0.0f ? r : 0.0f;
}

// ---------------------------------------------------------------- routing
// The live posting slots, compacted (in any order: routing keeps the nprobe
// smallest unique (distance, slot) keys, which does not depend on the order).
__global__ void k_live_idx(const uint8_t *live, uint32_t nb, uint32_t *out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
    if (live[b]) out[1 + atomicAdd(out, 1u)] = b;
}

// Query x live-posting-centroid distances, each pair summed in coordinate order
// with the rounding of seq_metric (so routing is unchanged), as a tiled
// kernel: a block covers 64 queries x 64 centroids, staged 32 dimensions at a
// time in shared memory (row-major, rows padded to 33 floats: coalesced,
// conflict-free staging and at most 2-way conflicts in the reads); each thread
// owns a 4 x 4 tile of pairs.  Zero padding beyond d adds +0 and leaves every
// sum unchanged.
constexpr int kRT = 64, kRD = 32, kRS = kRD + 1;
// Columns follow cidx[1 ..] (cidx[0] live postings; blocks past it exit),
// rows of D are ldd floats apart.
__global__ void __launch_bounds__(256) k_route(const float *__restrict__ Q, uint32_t nq, uint32_t qstride,
                                               const float *__restrict__ C, const uint32_t *__restrict__ cidx,
                                               uint32_t d, uint32_t dpad, int metric, float *__restrict__ D,
                                               uint32_t ldd) {
  __shared__ float qt[kRT * kRS];
  __shared__ float ct[kRT * kRS];
  __shared__ float qn[kRT], cn[kRT];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const uint32_t q0 = blockIdx.y * kRT, c0 = blockIdx.x * kRT;
  const uint32_t nb = __ldg(cidx);
  if (c0 >= nb) return;  // the whole block: fewer live postings than slots
  const uint32_t *col = cidx + 1;
  const bool l2 = metric == DG_L2SQ || metric == DG_L2;
  if (metric == DG_COSINE && threadIdx.x < 2 * kRT) {  // |q|^2, |c|^2 in coordinate order
    const int r = threadIdx.x & (kRT - 1);
    const bool isq = threadIdx.x < kRT;
    const uint32_t row = (isq ? q0 : c0) + r;
    float s2 = 0.0f;
    if (row < (isq ? nq : nb)) {
      const float *x = isq ? Q + (size_t)row * qstride : C + (size_t)col[row] * dpad;
      for (uint32_t i = 0; i < d; ++i) s2 = __fadd_rn(s2, __fmul_rn(x[i], x[i]));
    }
    (isq ? qn : cn)[r] = s2;
  }
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  for (uint32_t k0 = 0; k0 < dpad; k0 += kRD) {
    for (int e = threadIdx.x; e < kRT * kRD; e += 256) {
      const int r = e / kRD, k = e % kRD;
      const uint32_t kk = k0 + k;
      qt[r * kRS + k] = (q0 + r < nq && kk < d) ? Q[(size_t)(q0 + r) * qstride + kk] : 0.0f;
      ct[r * kRS + k] = (c0 + r < nb && kk < dpad) ? C[(size_t)col[c0 + r] * dpad + kk] : 0.0f;
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kRD; ++k) {
      float av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        av[i] = qt[(ty * 4 + i) * kRS + k];
        bv[i] = ct[(tx * 4 + i) * kRS + k];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (l2) {
            const float t = __fsub_rn(av[i], bv[j]);
            acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(t, t));
          } else {
            acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(av[i], bv[j]));
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t q = q0 + ty * 4 + i;
    if (q >= nq) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t c = c0 + tx * 4 + j;
      if (c >= nb) continue;
      const float a = acc[i][j];
      float v;
      if (metric == DG_L2SQ) v = a;
      else if (metric == DG_L2) v = __fsqrt_rn(a);
      else if (metric == DG_DOT) v = __fsub_rn(1.0f, a);
      else {
        const float aa = qn[ty * 4 + i], bb = cn[tx * 4 + j];
        if (aa == 0.0f && bb == 0.0f) v = 0.0f;
        else if (a == 0.0f) v = 1.0f;
        else {
          const float r = __fsub_rn(1.0f, __fdiv_rn(a, __fmul_rn(__fsqrt_rn(aa), __fsqrt_rn(bb))));
          v = r > 0.0f ? r : 0.0f;
        }
      }
      D[(size_t)q * ldd + c] = v;
    }
  }
}

// The reference's angular / dot from the three sums (RN intrinsics).
__device__ __forceinline__ float seq_finish(int met, float ab, float aa, float bb) {
  if (met == MET_DOT) return __fsub_rn(1.0f, ab);
  if (aa == 0.0f && bb == 0.0f) return 0.0f;
  if (ab == 0.0f) return 1.0f;
  const float r = __fsub_rn(1.0f, __fdiv_rn(ab, __fmul_rn(__fsqrt_rn(aa), __fsqrt_rn(bb))));
  return r > 0.0f ? r : 0.0f;
}

struct SpfLayout {
  uint32_t p0, p1, r0, r1, cst, qf, prov, total;
};
__host__ __device__ inline SpfLayout spf_layout(uint32_t pcap, uint32_t rcap, uint32_t dpad, int kind,
                                                uint32_t pq_M, uint32_t pq_K, uint32_t P) {
  SpfLayout L{};
  uint32_t o = 0;
  L.p0 = o; o += pcap * 8;
  L.p1 = o; o += pcap * 8;
  L.r0 = o; o += rcap * 8;
  L.r1 = o; o += rcap * 8;
  L.cst = o; o += 64 * 8;
  L.qf = o; o += align16(dpad * 4);
  L.prov = o;
  uint32_t p = 0;
  if (kind == SPF_PQ) p = pq_M * pq_K * 4;
  else if (kind == SPF_INT8) p = align16(dpad);
  else if (kind == SPF_F16) p = align16(dpad * 4);
  else if (kind == SPF_RABITQ) p = 4 * (P / 64) * 8 + 32 + align16(P * 4);  // also the decode buffer (P floats)
  o += align16(p);
  L.total = align16(o);
  return L;
}

__device__ __forceinline__ bool is_deleted(const uint32_t *bm, uint32_t id) {
  return (__ldg(bm + (id >> 5)) >> (id & 31)) & 1u;
}

// Distances of lane j's entry (row index `row` into the code array, valid for
// j < cnt) by the posting's code kind (quantized_distance_from_codes).
template <int KIND, int MET>
__device__ __forceinline__ float entry_distance(const SpfArgs &a, uint8_t *wsm, const SpfLayout &Ly, uint32_t row,
                                                int cnt, int lane, float qq) {
  const float *qs = reinterpret_cast<const float *>(wsm + Ly.qf);
  const bool sq = a.metric == DG_L2;
  if (KIND == SPF_RAW) {
    // code = the f32 vector: dist.eval(query, code)
    return rows_distance<8, 0, MET>(a.codes, a.code_stride, (a.code_stride / 16) / 8, qs, row, cnt, lane, sq, qq);
  } else if (KIND == SPF_F16) {
    const float *qx = MET == MET_L2 ? reinterpret_cast<const float *>(wsm + Ly.prov) : qs;
    const int ch = a.code_stride / 16;
    return ch % 8 == 0 ? rows_distance<8, 2, MET>(a.codes, a.code_stride, ch / 8, qx, row, cnt, lane, sq, qq)
                       : rows_distance<4, 2, MET>(a.codes, a.code_stride, ch / 4, qx, row, cnt, lane, sq, qq);
  } else if (KIND == SPF_INT8) {
    const int ch = a.code_stride / 16;
    if (MET == MET_L2) {
      const uint8_t *qc = wsm + Ly.prov;
      const uint32_t s = ch % 8 == 0 ? int8_l2_group<8>(a.codes, a.code_stride, ch / 8, qc, row, cnt, lane)
                         : ch % 4 == 0 ? int8_l2_group<4>(a.codes, a.code_stride, ch / 4, qc, row, cnt, lane)
                                       : int8_l2_group<2>(a.codes, a.code_stride, ch / 2, qc, row, cnt, lane);
      const float dd = __fmul_rn(__fmul_rn(__uint2float_rn(s), a.i8_scale), a.i8_scale);
      return sq ? __fsqrt_rn(dd) : dd;
    }
    return ch % 8 == 0 ? int8_decode_group<8, MET>(a.codes, a.code_stride, ch / 8, qs, a.i8_scale, a.i8_offset, a.d,
                                                   row, cnt, lane, qq)
         : ch % 4 == 0 ? int8_decode_group<4, MET>(a.codes, a.code_stride, ch / 4, qs, a.i8_scale, a.i8_offset, a.d,
                                                   row, cnt, lane, qq)
                       : int8_decode_group<2, MET>(a.codes, a.code_stride, ch / 2, qs, a.i8_scale, a.i8_offset, a.d,
                                                   row, cnt, lane, qq);
  } else if (KIND == SPF_PQ && MET == MET_L2) {
    const float *lut = reinterpret_cast<const float *>(wsm + Ly.prov);
    float dd = 0.0f;
    if (lane < cnt) {
      const uint8_t *crow = a.codes + (size_t)row * a.code_stride;
      const uint32_t K = a.pq_K;
      for (uint32_t m = 0; m < a.pq_M; ++m) dd = __fadd_rn(dd, lut[m * K + __ldg(crow + m)]);
    }
    return sq ? __fsqrt_rn(dd) : dd;
  } else if (KIND == SPF_PQ) {
    // cosine / dot: the metric of the decoded code (centroid concatenation,
    // src/pq.rs:151-160), summed in coordinate order as the reference's
    // metric does; one entry per lane
    float ab = 0.0f, bb = 0.0f;
    if (lane < cnt) {
      const uint8_t *crow = a.codes + (size_t)row * a.code_stride;
      for (uint32_t m = 0; m < a.pq_M; ++m) {
        const float *cen = a.pq_cb + ((size_t)m * a.pq_K + __ldg(crow + m)) * a.pq_ds;
        const float *qm = qs + m * a.pq_ds;
        for (uint32_t j = 0; j < a.pq_ds; ++j) {
          const float x = __ldg(cen + j);
          ab = __fadd_rn(ab, __fmul_rn(qm[j], x));
          bb = __fadd_rn(bb, __fmul_rn(x, x));
        }
      }
    }
    return seq_finish(MET, ab, qq, bb);
  } else {
    // RaBitQ with cosine / dot: decode against the posting centroid
    // (src/spfresh.rs:344-354, src/rabitq.rs:224-238), one entry at a time
    // across the warp: signs +-1/sqrt(P), three inverse rounds, c + |v-c| r.
    const uint32_t P = a.rq_padded;
    float *r = reinterpret_cast<float *>(wsm + Ly.prov);
    const float inv = __fdiv_rn(1.0f, __fsqrt_rn((float)P));
    const uint32_t b = row / a.cap;
    const float *cen = a.centroids + (size_t)b * a.dpad;
    float mine = 0.0f;
    for (int j = 0; j < cnt; ++j) {
      const uint32_t rj = __shfl_sync(kFull, row, j);
      const uint8_t *code = a.codes + (size_t)rj * a.code_stride;
      for (uint32_t i = lane; i < P; i += 32) r[i] = ((__ldg(code + (i >> 3)) >> (i & 7)) & 1u) ? inv : -inv;
      __syncwarp();
      for (int rd = 2; rd >= 0; --rd) {
        for (uint32_t h = 1; h < P; h *= 2) {
          for (uint32_t t = lane; t < P / 2; t += 32) {
            const uint32_t x0 = (t / h) * 2 * h + (t % h);
            const float u = r[x0], v = r[x0 + h];
            r[x0] = __fadd_rn(u, v);
            r[x0 + h] = __fsub_rn(u, v);
          }
          __syncwarp();
        }
        for (uint32_t i = lane; i < P; i += 32) r[i] = __fmul_rn(r[i], a.rq_signs[rd * P + i]);
        __syncwarp();
      }
      const float norm = __fsqrt_rn(__ldg(reinterpret_cast<const float *>(code + P / 8)));
      float ab = 0.0f, bb = 0.0f;
      for (uint32_t i = lane; i < a.d; i += 32) {
        const float o = __fadd_rn(__ldg(cen + i), __fmul_rn(norm, r[i]));
        ab = fmaf(qs[i], o, ab);
        bb = fmaf(o, o, bb);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ab += __shfl_xor_sync(kFull, ab, o);
        bb += __shfl_xor_sync(kFull, bb, o);
      }
      if (lane == j) mine = seq_finish(MET, ab, qq, bb);
      __syncwarp();
    }
    return mine;
  }
}

template <int KIND, int MET>
__global__ void __launch_bounds__(128, 4) spfresh_kernel(SpfArgs a, SpfLayout Ly, uint32_t pcap, uint32_t rcap) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *wsm = smem + (size_t)warp * Ly.total;
  uint64_t *const P[2] = {reinterpret_cast<uint64_t *>(wsm + Ly.p0), reinterpret_cast<uint64_t *>(wsm + Ly.p1)};
  uint64_t *const Rl[2] = {reinterpret_cast<uint64_t *>(wsm + Ly.r0), reinterpret_cast<uint64_t *>(wsm + Ly.r1)};
  uint64_t *cst = reinterpret_cast<uint64_t *>(wsm + Ly.cst);
  float *qs = reinterpret_cast<float *>(wsm + Ly.qf);
  while (true) {
    uint32_t q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1u);
    q = __shfl_sync(kFull, q, 0);
    if (q >= a.nq) break;
    const float *qg = a.Q + (size_t)q * a.d;
    for (uint32_t i = lane; i < a.dpad; i += 32) qs[i] = i < a.d ? qg[i] : 0.0f;
    __syncwarp();
    float qq = 0.0f;
    if (MET == MET_COS && (KIND == SPF_PQ || KIND == SPF_RABITQ)) {
      // |q|^2 in coordinate order, as the reference's angular()
      if (lane == 0)
        for (uint32_t i = 0; i < a.d; ++i) qq = __fadd_rn(qq, __fmul_rn(qs[i], qs[i]));
      qq = __shfl_sync(kFull, qq, 0);
    } else if (MET == MET_COS) {
      for (uint32_t i = lane; i < a.dpad; i += 32) qq = fmaf(qs[i], qs[i], qq);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) qq += __shfl_xor_sync(kFull, qq, o);
    }
    // ---- 1. routing
    const int nprobe = (int)max(a.nprobe, 1u);
    int pcur = 0, psize = 0;
    if (a.probe_in) {  // routed already (probes after the probe_ratio cut)
      psize = (int)a.probe_in_cnt[q];
      for (int i = lane; i < psize; i += 32) P[0][i] = make_key(0.0f, a.probe_in[(size_t)q * a.nprobe + i]);
      __syncwarp();
    } else if (a.route) {
      // precomputed distances: the loads of 8 batches go out before their
      // (in-order) insertions
      const float *rq = a.route + (size_t)q * a.nblocks;
      const uint32_t nl = __ldg(a.route_idx);
      const uint32_t *col = a.route_idx + 1;
      for (uint32_t j0 = 0; j0 < nl; j0 += 32 * 8) {
        uint64_t keys[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const uint32_t j = j0 + 32u * u + lane;
          keys[u] = j < nl ? make_key(__ldg(rq + j), __ldg(col + j)) : kKeyInvalid;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) insert_batch(keys[u], P, pcur, psize, nprobe, cst, lane);
      }
    } else {
      for (uint32_t b0 = 0; b0 < a.nblocks; b0 += 32) {
        const uint32_t b = b0 + lane;
        uint64_t key = kKeyInvalid;
        if (b < a.nblocks && a.live[b])
          key = make_key(seq_metric(qs, a.centroids + (size_t)b * a.dpad, a.d, a.metric), b);
        insert_batch(key, P, pcur, psize, nprobe, cst, lane);
      }
    }
    // ---- 2. probe_ratio cut
    int np = psize;
    if (np > 0 && isfinite(a.probe_ratio) && !a.probe_in) {
      const float d0 = key_dist(P[pcur][0]);
      if (d0 >= 0.0f) {
        const float lim = __fmul_rn(d0, fmaxf(a.probe_ratio, 1.0f));
        int first_out = psize;
        for (int i = lane; i < psize; i += 32)
          if (key_dist(P[pcur][i]) > lim) first_out = min(first_out, i);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) first_out = min(first_out, __shfl_xor_sync(kFull, first_out, o));
        np = first_out;
      }
    }
    if (a.probe_out) {  // posting-major scan: hand over the probed postings
      for (int i = lane; i < np; i += 32) a.probe_out[(size_t)q * a.nprobe + i] = key_id(P[pcur][i]);
      if (lane == 0) a.probe_cnt[q] = (uint32_t)np;
      __syncwarp();
      continue;
    }
    // ---- per-query code state
    if (KIND == SPF_PQ && MET == MET_L2) {
      SearchArgs sa{};
      sa.pq_M = a.pq_M;
      sa.pq_K = a.pq_K;
      sa.pq_ds = a.pq_ds;
      sa.pq_cb = a.pq_cb;
      build_pq_lut(sa, qs, reinterpret_cast<float *>(wsm + Ly.prov), lane);
    } else if (KIND == SPF_INT8) {
      uint8_t *qc8 = wsm + Ly.prov;
      const float inv = __fdiv_rn(1.0f, a.i8_scale);
      const float beta = __fdiv_rn(-a.i8_offset, a.i8_scale);
      for (uint32_t i = lane; i < a.dpad; i += 32) qc8[i] = i < a.d ? int8_code(qs[i], inv, beta) : 0;
    } else if (KIND == SPF_F16) {
      float *qh = reinterpret_cast<float *>(wsm + Ly.prov);
      for (uint32_t i = lane; i < a.dpad; i += 32) qh[i] = __half2float(__float2half_rn(qs[i]));
    }
    __syncwarp();
    const uint32_t k = a.k;
    int rcur = 0, rsize = 0;
    uint32_t *oids32 = nullptr;
    (void)oids32;
    if (KIND == SPF_RABITQ && MET == MET_L2) {
      // ---- 4. search_rabitq: heap of the k smallest exact distances
      const int kk = (int)k;
      uint8_t *pv = wsm + Ly.prov;
      uint64_t *planes = reinterpret_cast<uint64_t *>(pv);
      float *k5 = reinterpret_cast<float *>(pv + 4 * (a.rq_padded / 64) * 8);
      float *rbuf = reinterpret_cast<float *>(pv + 4 * (a.rq_padded / 64) * 8 + 32);
      const uint32_t P2 = a.rq_padded;
      for (int pi = 0; pi < np; ++pi) {
        const uint32_t b = key_id(P[pcur][pi]);
        rabitq_prepare(qs, a.d, P2, a.centroids + (size_t)b * a.dpad, a.rq_signs, rbuf, planes, k5, lane);
        const uint32_t n_e = a.len[b];
        for (uint32_t e0 = 0; e0 < n_e; e0 += 32) {
          const uint32_t e = e0 + lane;
          const uint32_t row = b * a.cap + e;
          bool valid = e < n_e;
          uint32_t id = valid ? __ldg(a.ids + row) : 0u;
          if (valid && is_deleted(a.deleted, id)) valid = false;
          float est = 0.0f, err = 0.0f;
          if (valid) {
            const uint8_t *code = a.codes + (size_t)row * a.code_stride;
            est = rabitq_est(code, P2, planes, k5);
            const float2 nf = __ldg(reinterpret_cast<const float2 *>(code + P2 / 8));
            const float ip = nf.y > 0.0f ? __fdiv_rn(__fsqrt_rn(nf.x), nf.y) : 0.0f;
            err = ip > 0.0f ? __fmul_rn(__fmul_rn(__fmul_rn(k5[1], nf.y), 1.9f),
                                        __fsqrt_rn(__fdiv_rn(fmaxf(__fsub_rn(1.0f, __fmul_rn(ip, ip)), 0.0f),
                                                             __fsub_rn((float)P2, 1.0f))))
                            : __int_as_float(0x7f800000);
          }
          // candidates that pass against the threshold at the start of the batch
          // (the threshold only falls, so nothing else can pass later)
          const float kth0 = rsize < kk ? __int_as_float(0x7f800000) : key_dist(Rl[rcur][kk - 1]);
          const bool maybe = valid && __fsub_rn(est, err) < kth0;
          const uint32_t mm = __ballot_sync(kFull, maybe);
          if (!mm) continue;
          // exact squared distances of those, computed together
          uint32_t *stage = reinterpret_cast<uint32_t *>(cst);
          if (maybe) stage[__popc(mm & lanemask_lt(lane))] = id;
          __syncwarp();
          const int cnt = __popc(mm);
          const uint32_t cid = lane < cnt ? stage[lane] : 0u;
          const float ex = rows_distance<8, 0, MET_L2>(reinterpret_cast<const uint8_t *>(a.raw), a.dpad * 4,
                                                       (a.dpad / 4) / 8, qs, cid, cnt, lane, false, 0.0f);
          __syncwarp();
          // replay in entry order against the running threshold
          int slot = 0;
          for (int j = 0; j < 32; ++j) {
            if (!((mm >> j) & 1u)) continue;
            const float ej = __shfl_sync(kFull, __fsub_rn(est, err), j);
            const float xj = __shfl_sync(kFull, ex, slot);
            const uint32_t ij = __shfl_sync(kFull, id, j);
            ++slot;
            const float kth = rsize < kk ? __int_as_float(0x7f800000) : key_dist(Rl[rcur][kk - 1]);
            if (ej < kth) insert_batch(lane == 0 ? make_key(xj, ij) : kKeyInvalid, Rl, rcur, rsize, kk, cst + 32, lane);
          }
        }
      }
      // sqrt for DistL2, then (distance, id) order
      uint64_t *tmp = Rl[rcur ^ 1];
      for (int i = lane; i < rsize; i += 32) {
        const uint64_t kv = Rl[rcur][i];
        const float dd = key_dist(kv);
        tmp[i] = make_key(a.metric == DG_L2 ? __fsqrt_rn(dd) : dd, key_id(kv));
      }
      __syncwarp();
      warp_sort_smem(tmp, rsize, lane);
      const int count = min(rsize, kk);
      for (int i = lane; i < (int)k; i += 32) {
        a.out_ids[(size_t)q * k + i] = i < count ? (uint64_t)key_id(tmp[i]) : DG_PAD64;
        a.out_d[(size_t)q * k + i] = i < count ? key_dist(tmp[i]) : __int_as_float(0x7f800000);
      }
      if (lane == 0) a.out_cnt[q] = (uint32_t)count;
      __syncwarp();
      continue;
    }
    // ---- 3. scan (src/spfresh.rs:702-717)
    const bool rerank = KIND != SPF_RAW && a.rerank > 0;
    const int want = (int)(rerank ? max(k, a.rerank) : k);
    for (int pi = 0; pi < np; ++pi) {
      const uint32_t b = key_id(P[pcur][pi]);
      const uint32_t n_e = a.len[b];
      for (uint32_t e0 = 0; e0 < n_e; e0 += 32) {
        const uint32_t e = e0 + lane;
        const int cnt = (int)min(32u, n_e - e0);
        const uint32_t row = b * a.cap + min(e, n_e - 1);
        const uint32_t id = __ldg(a.ids + row);
        const float dd = entry_distance<KIND, MET>(a, wsm, Ly, row, cnt, lane, qq);
        const bool ok = e < n_e && !is_deleted(a.deleted, id);
        insert_batch(ok ? make_key(dd, id) : kKeyInvalid, Rl, rcur, rsize, want, cst, lane);
      }
    }
    // rerank from the raw store (src/spfresh.rs:719-723), then (distance, id) order
    uint64_t *src = Rl[rcur];
    uint64_t *tmp = Rl[rcur ^ 1];
    if (rerank) {
      for (int g0 = 0; g0 < rsize; g0 += 32) {
        const int cnt = min(32, rsize - g0);
        const uint32_t cid = lane < cnt ? key_id(src[g0 + lane]) : 0u;
        float ex = 0.0f;
        if (MET == MET_L2)
          ex = rows_distance<8, 0, MET_L2>(reinterpret_cast<const uint8_t *>(a.raw), a.dpad * 4, (a.dpad / 4) / 8, qs,
                                           cid, cnt, lane, a.metric == DG_L2, qq);
        else
          ex = rows_distance<8, 0, MET>(reinterpret_cast<const uint8_t *>(a.raw), a.dpad * 4, (a.dpad / 4) / 8, qs,
                                        cid, cnt, lane, false, qq);
        if (lane < cnt) tmp[g0 + lane] = make_key(ex, cid);
      }
      __syncwarp();
      warp_sort_smem(tmp, rsize, lane);
      src = tmp;
    }
    const int count = min(rsize, (int)k);
    for (int i = lane; i < (int)k; i += 32) {
      a.out_ids[(size_t)q * k + i] = i < count ? (uint64_t)key_id(src[i]) : DG_PAD64;
      a.out_d[(size_t)q * k + i] = i < count ? key_dist(src[i]) : __int_as_float(0x7f800000);
    }
    if (lane == 0) a.out_cnt[q] = (uint32_t)count;
    __syncwarp();
  }
}

template <int KIND, int MET>
static DgStatus spf_launch(const SpfArgs &a, uint32_t pcap, uint32_t rcap, cudaStream_t st) {
  const SpfLayout Ly = spf_layout(pcap, rcap, a.dpad, KIND, a.pq_M, a.pq_K, a.rq_padded);
  auto kern = spfresh_kernel<KIND, MET>;
  const uint32_t smem = Ly.total * 4;
  int dev = 0, sms = 0, optin = 0;
  DG_CUDA(cudaGetDevice(&dev));
  DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem > (uint32_t)optin) return fail(DG_ENOTSUP, "SPFresh search state does not fit in shared memory");
  DG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int nb = 0;
  DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 128, smem));
  if (nb < 1) return fail(DG_ENOTSUP, "SPFresh kernel cannot be resident");
  const int grid = std::max(1, std::min(nb * sms, (int)((a.nq + 3) / 4)));
  kern<<<grid, 128, smem, st>>>(a, Ly, pcap, rcap);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// ------------------------------------------------ posting-major scan (raw f32, L2)
// A batch probes each posting from many queries (10k queries x 64 probes over
// 24k postings: ~27 each).  Instead of every query reading its postings, the
// (query, posting) pairs are grouped by posting and one CTA loads a posting's
// entries into shared memory once and scores every query that probes it,
// keeping each pair's k best; a per-query merge then forms the result.  The
// result is the k smallest (distance, id) keys over the live entries of the
// probed postings, as the query-major scan (src/spfresh.rs:702-727); each
// distance is |q|^2 + |x|^2 - 2 q.x with FP32 FMA sums (exact on
// integer-valued data, within FP32 rounding otherwise).
constexpr int kPmQ = 32;   // queries per work item
constexpr int kPmT = 64;   // entries per shared-memory tile
constexpr int kPmK = 64;   // largest k of the posting-major scan

// Radix pass of k_pm_select: among this warp's keys matching (prefix, mask),
// counts `width` bits at `shift`, then finds the bucket holding the need-th
// key.  Returns that bucket; need becomes its rank inside the bucket.
template <typename KeyOf>
__device__ __forceinline__ uint32_t pm_radix_pass(uint32_t *hist, uint32_t nl, KeyOf key_of, uint32_t prefix,
                                                  uint32_t mask, int shift, int width, uint32_t &need, int lane) {
  const uint32_t nb = 1u << width;
  for (uint32_t i = lane; i < nb; i += 32) hist[i] = 0u;
  __syncwarp();
  for (uint32_t j = lane; j < nl; j += 32) {
    bool ok;
    const uint32_t v = key_of(j, ok);
    if (ok && (v & mask) == prefix) atomicAdd(hist + ((v >> shift) & (nb - 1)), 1u);
  }
  __syncwarp();
  // each lane sums nb / 32 consecutive buckets; a warp scan of the sums
  const uint32_t per = nb / 32;
  uint32_t sum = 0;
  for (uint32_t i = 0; i < per; ++i) sum += hist[lane * per + i];
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t excl = incl - sum;
  const uint32_t owner = __ffs(__ballot_sync(kFull, incl >= need)) - 1;
  uint32_t bucket = 0, below = 0;
  if (lane == (int)owner) {
    uint32_t c = excl;
    for (uint32_t i = 0; i < per; ++i) {
      const uint32_t h = hist[lane * per + i];
      if (c + h >= need) {
        bucket = lane * per + i;
        below = c;
        break;
      }
      c += h;
    }
  }
  bucket = __shfl_sync(kFull, bucket, owner);
  below = __shfl_sync(kFull, below, owner);
  need -= below;
  __syncwarp();
  return bucket;
}

// The posting-major scan's probes: per query (one warp) the exact set of the
// nprobe smallest (distance, slot) keys of its routing row -- the set the
// query-major kernel's sorted selection holds (src/spfresh.rs:358-378) -- by
// radix select over the distance bits (three passes; distances are >= 0 under
// L2, so their bits order as the values) and, for keys equal to the cut-off
// distance, over the slot numbers (two passes), then the probe_ratio cut
// (:690-700).  Unordered output.
__global__ void __launch_bounds__(128) k_pm_select(const float *route, const uint32_t *route_idx, uint32_t nq,
                                                   uint32_t nblocks, uint32_t nprobe, float probe_ratio,
                                                   uint32_t *probe_out, uint32_t *probe_cnt) {
  __shared__ uint32_t hist_all[4][2048];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t *hist = hist_all[warp];
  const uint32_t nl = __ldg(route_idx);
  const uint32_t *col = route_idx + 1;
  for (uint32_t q = blockIdx.x * 4 + warp; q < nq; q += gridDim.x * 4) {
    const float *rq = route + (size_t)q * nblocks;
    const uint32_t take = min(nprobe, nl);
    // the nearest distance, for the probe_ratio cut, and a column holding it
    float d0 = __int_as_float(0x7f800000);
    uint32_t j0min = 0xffffffffu;
    for (uint32_t j = lane; j < nl; j += 32) {
      const float v = __ldg(rq + j);
      if (v < d0) {
        d0 = v;
        j0min = j;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float od = __shfl_xor_sync(kFull, d0, o);
      const uint32_t oj = __shfl_xor_sync(kFull, j0min, o);
      if (od < d0 || (od == d0 && oj < j0min)) {
        d0 = od;
        j0min = oj;
      }
    }
    uint32_t tbits = 0xffffffffu, tslot = 0xffffffffu;  // cut-off key (all keys when take == nl)
    if (take > 0 && take < nl) {
      uint32_t need = take, prefix = 0, mask = 0;
      auto dist_bits = [&](uint32_t j, bool &ok) {
        ok = true;
        return __float_as_uint(__ldg(rq + j));
      };
      const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
      for (int ps = 0; ps < 3; ++ps) {
        const uint32_t b = pm_radix_pass(hist, nl, dist_bits, prefix, mask, shifts[ps], widths[ps], need, lane);
        prefix |= b << shifts[ps];
        mask |= ((1u << widths[ps]) - 1u) << shifts[ps];
      }
      tbits = prefix;  // `need` keys at exactly this distance are taken, the smallest slots first
      auto tie_slot = [&](uint32_t j, bool &ok) {
        ok = __float_as_uint(__ldg(rq + j)) == tbits;
        return __ldg(col + j);
      };
      uint32_t sp = 0, sm = 0;
      const int ts[2] = {11, 0}, tw[2] = {11, 11};
      for (int ps = 0; ps < 2; ++ps) {
        const uint32_t b = pm_radix_pass(hist, nl, tie_slot, sp, sm, ts[ps], tw[ps], need, lane);
        sp |= b << ts[ps];
        sm |= ((1u << tw[ps]) - 1u) << ts[ps];
      }
      tslot = sp;
    }
    const bool cut = isfinite(probe_ratio) && d0 >= 0.0f;
    const float lim = cut ? __fmul_rn(d0, fmaxf(probe_ratio, 1.0f)) : __int_as_float(0x7f800000);
    uint32_t n_out = 0, near_at = 0;
    for (uint32_t j0 = 0; j0 < nl; j0 += 32) {
      const uint32_t j = j0 + lane;
      bool sel = false;
      uint32_t slot = 0;
      if (j < nl) {
        const float dv = __ldg(rq + j);
        const uint32_t bits = __float_as_uint(dv);
        slot = __ldg(col + j);
        sel = (bits < tbits || (bits == tbits && slot <= tslot)) && !(dv > lim);
      }
      const uint32_t m = __ballot_sync(kFull, sel);
      const uint32_t at = n_out + __popc(m & lanemask_lt(lane));
      if (sel) probe_out[(size_t)q * nprobe + at] = slot;
      const uint32_t hm = __ballot_sync(kFull, sel && j == j0min);
      if (hm) near_at = __shfl_sync(kFull, at, __ffs(hm) - 1);
      n_out += __popc(m);
    }
    __syncwarp();
    // the nearest probe first (the posting-major bound starts from it; the
    // scan does not depend on the order of the probes)
    if (lane == 0 && near_at > 0 && near_at < n_out) {
      uint32_t *po = probe_out + (size_t)q * nprobe;
      const uint32_t t = po[0];
      po[0] = po[near_at];
      po[near_at] = t;
    }
    if (lane == 0) probe_cnt[q] = n_out;
    __syncwarp();
  }
}

__global__ void k_pm_count(const uint32_t *probe, const uint32_t *cnt, uint32_t nq, uint32_t nprobe,
                           uint32_t *pcount) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < (uint64_t)nq * nprobe;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t q = (uint32_t)(t / nprobe), i = (uint32_t)(t % nprobe);
    if (i < cnt[q]) atomicAdd(pcount + probe[t], 1u);
  }
}

// Exclusive scans of pcount (pair starts) and of ceil(pcount / kPmQ) (item
// starts) over nb postings; out[nb] of each receives the total.  One block.
__global__ void __launch_bounds__(1024) k_pm_scan(const uint32_t *pcount, uint32_t nb, uint32_t *pstart,
                                                  uint32_t *istart) {
  __shared__ uint32_t sp[1024], si[1024];
  const uint32_t t = threadIdx.x, per = (nb + 1023) / 1024;
  const uint32_t b0 = min(nb, t * per), b1 = min(nb, b0 + per);
  uint32_t a = 0, c = 0;
  for (uint32_t b = b0; b < b1; ++b) {
    a += pcount[b];
    c += (pcount[b] + kPmQ - 1) / kPmQ;
  }
  sp[t] = a;
  si[t] = c;
  __syncthreads();
  for (uint32_t o = 1; o < 1024; o <<= 1) {
    const uint32_t va = t >= o ? sp[t - o] : 0u, vc = t >= o ? si[t - o] : 0u;
    __syncthreads();
    sp[t] += va;
    si[t] += vc;
    __syncthreads();
  }
  a = sp[t] - a;  // exclusive prefix of this thread's range
  c = si[t] - c;
  for (uint32_t b = b0; b < b1; ++b) {
    pstart[b] = a;
    istart[b] = c;
    a += pcount[b];
    c += (pcount[b] + kPmQ - 1) / kPmQ;
  }
  if (t == 1023) {
    pstart[nb] = sp[1023];
    istart[nb] = si[1023];
  }
}

__global__ void k_pm_scatter(const uint32_t *probe, const uint32_t *cnt, uint32_t nq, uint32_t nprobe,
                             const uint32_t *pstart, uint32_t *pfill, uint32_t *pair_q, uint32_t *pos_of) {
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < (uint64_t)nq * nprobe;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t q = (uint32_t)(t / nprobe), i = (uint32_t)(t % nprobe);
    if (i >= cnt[q]) continue;
    const uint32_t b = probe[t];
    const uint32_t pos = pstart[b] + atomicAdd(pfill + b, 1u);
    pair_q[pos] = q;
    pos_of[t] = pos;
  }
}

// items: (posting, first pair, pair count <= kPmQ)
__global__ void k_pm_items(const uint32_t *pcount, const uint32_t *pstart, const uint32_t *istart, uint32_t nb,
                           uint4 *items) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const uint32_t c = pcount[b];
    for (uint32_t j = 0; j * kPmQ < c; ++j)
      items[istart[b] + j] = make_uint4(b, pstart[b] + j * kPmQ, min((uint32_t)kPmQ, c - j * kPmQ), 0u);
  }
}

// Tensor-core form of the tile's dot products.  Integer-valued rows and
// queries with |x| <= 2048 are exact in FP16, every FP16 x FP16 product is
// exact in FP32, and when every partial sum stays below 2^24 (d * max|q| *
// max|x| < 2^24) the FP32 accumulation is exact too: the tensor cores then
// return the dot products of the FMA chain below bit for bit.  A tile or a query set outside those
// bounds takes the FMA chain.
constexpr float kPmExactSum = 16777216.0f;  // 2^24
constexpr float kPmF16Int = 2048.0f;        // integers up to this magnitude are exact in FP16

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}

__device__ __forceinline__ void mma_f16_16x8x16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// FP16 bits of x and whether x is an integer exact in FP16 (|x| <= 2048).
__device__ __forceinline__ uint16_t f16_exact(float x, bool &ok) {
  ok = x == rintf(x) && fabsf(x) <= kPmF16Int;
  return __half_as_ushort(__float2half_rn(x));
}

// Shared-memory row stride (in FP16 elements) of the converted copies: dk + 8,
// so that the eight 16-byte rows one ldmatrix reads fall in distinct banks.
__host__ __device__ inline uint32_t pm_ks(uint32_t d) { return ((d + 15u) & ~15u) + 8u; }
// Capacity of a pair's k-best list: k rounded up to 16 (at most kPmK), which
// keeps the scan's shared memory at three CTAs per SM for d = 96, k <= 16.
__host__ __device__ inline uint32_t pm_kcap(uint32_t k) { return (k + 15u) & ~15u; }

// One CTA (8 warps) per work item at a time: the item's queries and a tile of
// the posting's entries in shared memory; warp w scores queries w, w+8, ...
// against two entries per lane and keeps each query's k best.  The dot
// products of a tile come from the tensor cores (the warps split the 64 x 32
// tile into 16 x 16 blocks) when the tile and the queries meet the exactness
// bounds above, else from an FMA chain per pair.
// qthr[q] for each query of a posting-major chunk (a warp each): an upper
// bound of the query's k-th smallest scan distance, from the live entries of
// its first probe (the nearest one).  B, the k-th smallest of their
// coordinate-order squared distances, is within (d + 2) 2^-24 B of the exact
// value; the scan's |q|^2 + |x|^2 - 2 q.x differs from the exact value by at
// most (2d + 6) 2^-24 (|q|^2 + |x|^2).  So
//     B (1 + (d + 2) 2^-23) + 4 (d + 4) 2^-24 (|q|^2 + max |x|^2)
// (rounded up; its square root, rounded up, for euclidean) bounds the k-th
// smallest scan distance over the probes.  All ones when the first probe has
// fewer than k live entries.
__global__ void __launch_bounds__(128) k_pm_bound(SpfArgs a, const uint32_t *probe, const uint32_t *pcnt,
                                                  uint32_t nprobe, uint32_t k, uint32_t *qthr) {
  extern __shared__ float bsm[];  // [4][cap] squared distances
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *sv = bsm + (size_t)warp * a.cap;
  for (uint32_t q = blockIdx.x * 4 + warp; q < a.nq; q += gridDim.x * 4) {
    uint32_t tb = 0xffffffffu;
    if (pcnt[q] > 0) {
      const uint32_t b = probe[(size_t)q * nprobe];
      const uint32_t n_e = min(a.len[b], a.cap);
      const float *qg = a.Q + (size_t)q * a.d;
      float qq = 0.0f, xxm = 0.0f;
      for (uint32_t i = lane; i < a.d; i += 32) qq = fmaf(__ldg(qg + i), __ldg(qg + i), qq);
      int live = 0;
      for (uint32_t e0 = 0; e0 < n_e; e0 += 32) {
        const uint32_t e = e0 + lane;
        const bool ok = e < n_e && !is_deleted(a.deleted, __ldg(a.ids + (size_t)b * a.cap + e));
        float sd = 0.0f, xx = 0.0f;
        if (ok) {
          const float *x = reinterpret_cast<const float *>(a.codes + ((size_t)b * a.cap + e) * a.code_stride);
#pragma unroll 8
          for (uint32_t i = 0; i < a.d; ++i) {
            const float xv = __ldg(x + i), t = __fsub_rn(__ldg(qg + i), xv);
            sd = __fadd_rn(sd, __fmul_rn(t, t));
            xx = fmaf(xv, xv, xx);
          }
        }
        const uint32_t msk = __ballot_sync(kFull, ok);
        if (ok) sv[live + __popc(msk & lanemask_lt(lane))] = sd;
        live += __popc(msk);
        xxm = fmaxf(xxm, xx);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        qq += __shfl_xor_sync(kFull, qq, o);
        xxm = fmaxf(xxm, __shfl_xor_sync(kFull, xxm, o));
      }
      __syncwarp();
      if (live >= (int)k) {
        uint32_t lo = 0, hi = 0xffffffffu;  // the k-th smallest: smallest v with #{ <= v} >= k
        while (lo < hi) {
          const uint32_t mid = lo + ((hi - lo) >> 1);
          uint32_t c = 0;
          for (int i = lane; i < live; i += 32) c += ordered_bits(sv[i]) <= mid ? 1u : 0u;
          c = __reduce_add_sync(kFull, c);
          if (c >= k) hi = mid;
          else lo = mid + 1;
        }
        const float fd = (float)a.d;
        const float c1 = __fmul_ru(fd + 2.0f, 1.1920928955078125e-7f);  // (d + 2) 2^-23
        const float c2 = __fmul_ru(4.0f * (fd + 4.0f), 5.9604644775390625e-8f);  // 4 (d + 4) 2^-24
        float bound = __fadd_ru(__fmul_ru(ordered_float(lo), __fadd_ru(1.0f, c1)), __fmul_ru(c2, __fadd_ru(qq, xxm)));
        if (a.metric == DG_L2) bound = __fsqrt_ru(bound);
        tb = ordered_bits(bound);
      }
      __syncwarp();
    }
    if (lane == 0) qthr[q] = tb;
    __syncwarp();
  }
}

// qthr[q] (ordered distance bits) is an upper bound of query q's final k-th
// distance: k_pm_bound's, lowered to the k-th distance of any of its pair
// lists that holds k keys.  Entries farther than it cannot reach the result, so
// they are dropped before the pair-list insertion (keys at the bound stay,
// ties included); the result does not depend on when bounds arrive.
__global__ void __launch_bounds__(256) k_pm_scan_postings(SpfArgs a, const uint4 *items, const uint32_t *n_items,
                                                          uint32_t *item_counter, const uint32_t *pair_q,
                                                          uint64_t *pair_keys, uint32_t *pair_cnt, uint32_t k,
                                                          uint32_t *qthr) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // query rows dpad floats; tile rows d + 4 floats: 16-byte rows whose float4
  // columns fall in distinct banks within each quarter warp
  const uint32_t dq = a.dpad, dt = a.d + 4, d4 = a.d / 4;
  const uint32_t ks = pm_ks(a.d), dk = ks - 8, kc = pm_kcap(k);
  float *qsm = reinterpret_cast<float *>(smem);                              // [kPmQ][dpad]
  float *tile = qsm + kPmQ * dq;                                             // [kPmT][d + 4]
  uint32_t *tid = reinterpret_cast<uint32_t *>(tile + kPmT * dt);            // [kPmT] ids
  float *xn = reinterpret_cast<float *>(tid + kPmT);                         // [kPmT] |x|^2
  float *qn = xn + kPmT;                                                     // [kPmQ] |q|^2
  uint64_t *lists = reinterpret_cast<uint64_t *>(qn + kPmQ);                 // [kPmQ][2][kc]
  uint64_t *cst = lists + (size_t)kPmQ * 2 * kc;                             // [8][32]
  uint16_t *qh = reinterpret_cast<uint16_t *>(cst + 8 * 32);                 // [kPmQ][ks] FP16 queries
  uint16_t *th = qh + kPmQ * ks;                                             // [kPmT][ks] FP16 tile
  // [kPmQ][kPmT] tensor-core dot products, over the f32 tile once it is converted
  float *dm = tile;
  __shared__ uint32_t s_item, s_qbad, s_tbad, s_qmax, s_tmax;
  const uint32_t total = *n_items;
  const bool sq = a.metric == DG_L2;
  const uint32_t qh_s = (uint32_t)__cvta_generic_to_shared(qh), th_s = (uint32_t)__cvta_generic_to_shared(th);
  while (true) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(item_counter, 1u);
      s_qbad = 0u;
      s_qmax = 0u;
    }
    __syncthreads();
    const uint32_t it = s_item;
    __syncthreads();
    if (it >= total) break;
    const uint4 item = items[it];
    const uint32_t b = item.x, p0 = item.y, m = item.z;
    {  // queries: f32 rows (zero padded to dpad) and FP16 rows (zero padded to dk, rows past m zero)
      bool bad = false;
      float mx = 0.0f;
      for (uint32_t t = threadIdx.x; t < kPmQ * dk; t += blockDim.x) {
        const uint32_t j = t / dk, i = t % dk;
        const float x = (j < m && i < a.d) ? __ldg(a.Q + (size_t)pair_q[p0 + j] * a.d + i) : 0.0f;
        bool ok;
        qh[j * ks + i] = f16_exact(x, ok);
        bad |= !ok;
        mx = fmaxf(mx, fabsf(x));
        if (j < m && i < dq) qsm[j * dq + i] = x;
      }
      for (uint32_t t = threadIdx.x; t < m * dq; t += blockDim.x)
        if (t % dq >= dk) qsm[t] = 0.0f;  // dpad beyond the FP16 width
      if (__syncthreads_or(bad) && threadIdx.x == 0) s_qbad = 1u;
      if (mx > 0.0f) atomicMax(&s_qmax, __float_as_uint(mx));
    }
    __syncthreads();
    // query norms: a warp per query, lanes over the coordinates
    for (uint32_t j = warp; j < m; j += blockDim.x >> 5) {
      float s2 = 0.0f;
      for (uint32_t i = lane; i < a.d; i += 32) s2 = fmaf(qsm[j * dq + i], qsm[j * dq + i], s2);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(kFull, s2, o);
      if (lane == 0) qn[j] = s2;
    }
    // this warp's queries: j = warp + 8 u (u < 4)
    int cur[4] = {0, 0, 0, 0}, size[4] = {0, 0, 0, 0};
    const uint32_t n_e = a.len[b];
    for (uint32_t e0 = 0; e0 < n_e; e0 += kPmT) {
      const uint32_t ne = min((uint32_t)kPmT, n_e - e0);
      __syncthreads();  // the previous tile is consumed (and the queries are in place)
      if (threadIdx.x == 0) {
        s_tbad = 0u;
        s_tmax = 0u;
      }
      {  // the tile: f32 rows and FP16 rows (rows past ne and columns past d are zero)
        bool bad = false;
        float mx = 0.0f;
        const uint32_t k4 = dk / 4;
        for (uint32_t t = threadIdx.x; t < kPmT * k4; t += blockDim.x) {
          const uint32_t r = t / k4, c = t % k4;
          float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          if (r < ne && c < d4) {
            v = __ldg(reinterpret_cast<const float4 *>(a.codes + (size_t)(b * a.cap + e0 + r) * a.code_stride) + c);
            reinterpret_cast<float4 *>(tile + r * dt)[c] = v;
          }
          bool o0, o1, o2, o3;
          const uint32_t lo = f16_exact(v.x, o0) | ((uint32_t)f16_exact(v.y, o1) << 16);
          const uint32_t hi = f16_exact(v.z, o2) | ((uint32_t)f16_exact(v.w, o3) << 16);
          *reinterpret_cast<uint2 *>(th + r * ks + 4 * c) = make_uint2(lo, hi);
          bad |= !(o0 && o1 && o2 && o3);
          mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
        }
        for (uint32_t r = threadIdx.x; r < kPmT; r += blockDim.x) {
          uint32_t id = DG_PAD;
          if (r < ne) {
            id = __ldg(a.ids + b * a.cap + e0 + r);
            if (is_deleted(a.deleted, id)) id = DG_PAD;
          }
          tid[r] = id;
        }
        if (__syncthreads_or(bad) && threadIdx.x == 0) s_tbad = 1u;
        if (mx > 0.0f) atomicMax(&s_tmax, __float_as_uint(mx));
      }
      __syncthreads();
      // entry norms: four lanes per row (8 rows per warp pass), interleaved
      // coordinates, so a quarter warp reads one row's consecutive words
      for (uint32_t r0 = 8u * warp; r0 < ne; r0 += 8u * (blockDim.x >> 5)) {
        const uint32_t r = r0 + (lane >> 2);
        float s2 = 0.0f;
        if (r < ne)
          for (uint32_t i = lane & 3; i < a.d; i += 4) s2 = fmaf(tile[r * dt + i], tile[r * dt + i], s2);
        s2 += __shfl_xor_sync(kFull, s2, 1);
        s2 += __shfl_xor_sync(kFull, s2, 2);
        if (r < ne && (lane & 3) == 0) xn[r] = s2;
      }
      const float qm = __uint_as_float(s_qmax), tm = __uint_as_float(s_tmax);
      // (the dot products overwrite the f32 tile, which must hold kPmQ x kPmT floats)
      const bool tc = !s_qbad && !s_tbad && dt >= (uint32_t)kPmQ && (float)a.d * qm * tm < kPmExactSum;
      __syncthreads();  // xn read the f32 tile
      float acc[4][2];
#pragma unroll
      for (int u = 0; u < 4; ++u) acc[u][0] = acc[u][1] = 0.0f;
      if (tc) {
        // warp w: entries 16 (w % 4) .. +15 against queries 16 (w / 4) .. +15
        const uint32_t e16 = 16u * (warp & 3), q16 = 16u * (warp >> 2);
        float c[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
        const uint32_t arow = e16 + (lane & 15), acol = (lane >> 4) * 8;
        const uint32_t brow = q16 + (lane >> 4) * 8 + (lane & 7), bcol = ((lane >> 3) & 1) * 8;
        for (uint32_t k0 = 0; k0 < dk; k0 += 16) {
          uint32_t av[4], bv[4];
          ldsm_x4(av, th_s + 2u * (arow * ks + k0 + acol));
          ldsm_x4(bv, qh_s + 2u * (brow * ks + k0 + bcol));
          mma_f16_16x8x16(c[0], av, bv[0], bv[1]);
          mma_f16_16x8x16(c[1], av, bv[2], bv[3]);
        }
        // lane (g, t) holds entries g, g + 8 x queries 2t, 2t + 1 of each 8-query tile
        const uint32_t g = lane >> 2, t2 = 2 * (lane & 3);
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const uint32_t qc = q16 + 8 * nt + t2;
          dm[qc * kPmT + e16 + g] = c[nt][0];
          dm[(qc + 1) * kPmT + e16 + g] = c[nt][1];
          dm[qc * kPmT + e16 + g + 8] = c[nt][2];
          dm[(qc + 1) * kPmT + e16 + g + 8] = c[nt][3];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const uint32_t j = warp + 8 * u;
          acc[u][0] = dm[j * kPmT + lane];
          acc[u][1] = dm[j * kPmT + lane + 32];
        }
      } else {
        const float4 *e0p = reinterpret_cast<const float4 *>(tile + (size_t)lane * dt);
        const float4 *e1p = reinterpret_cast<const float4 *>(tile + (size_t)(lane + 32) * dt);
#pragma unroll 2
        for (uint32_t c = 0; c < d4; ++c) {
          const float4 x0 = e0p[c], x1 = e1p[c];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const uint32_t j = warp + 8 * u;
            if (j < m) {
              const float4 qv = reinterpret_cast<const float4 *>(qsm + j * dq)[c];
              acc[u][0] = fmaf(qv.w, x0.w, fmaf(qv.z, x0.z, fmaf(qv.y, x0.y, fmaf(qv.x, x0.x, acc[u][0]))));
              acc[u][1] = fmaf(qv.w, x1.w, fmaf(qv.z, x1.z, fmaf(qv.y, x1.y, fmaf(qv.x, x1.x, acc[u][1]))));
            }
          }
        }
      }
      const uint32_t id0 = tid[lane], id1 = tid[lane + 32];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const uint32_t j = warp + 8 * u;
        if (j >= m) continue;  // warp-uniform
        uint64_t *const bufs[2] = {lists + (size_t)j * 2 * kc, lists + (size_t)j * 2 * kc + kc};
        uint32_t *qt = qthr + pair_q[p0 + j];
        const uint32_t tb = *reinterpret_cast<volatile uint32_t *>(qt);
        // |q - x|^2 = |q|^2 + |x|^2 - 2 q.x (exact on integer-valued data)
        const float qq = qn[j];
        const float s0 = fmaxf(__fsub_rn(__fadd_rn(qq, xn[lane]), __fmul_rn(2.0f, acc[u][0])), 0.0f);
        const float s1 = fmaxf(__fsub_rn(__fadd_rn(qq, xn[lane + 32]), __fmul_rn(2.0f, acc[u][1])), 0.0f);
        const float d0 = sq ? __fsqrt_rn(s0) : s0, d1 = sq ? __fsqrt_rn(s1) : s1;
        const bool k0 = id0 != DG_PAD && ordered_bits(d0) <= tb, k1 = id1 != DG_PAD && ordered_bits(d1) <= tb;
        insert_batch(k0 ? make_key(d0, id0) : kKeyInvalid, bufs, cur[u], size[u], (int)k, cst + warp * 32, lane);
        insert_batch(k1 ? make_key(d1, id1) : kKeyInvalid, bufs, cur[u], size[u], (int)k, cst + warp * 32, lane);
        if (size[u] >= (int)k && lane == 0) {
          const uint32_t nb = key_hi(bufs[cur[u]][k - 1]);
          if (nb < tb) atomicMin(qt, nb);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t j = warp + 8 * u;
      if (j >= m) continue;
      const uint64_t *lst = lists + (size_t)j * 2 * kc + (size_t)cur[u] * kc;
      for (int i = lane; i < size[u]; i += 32) pair_keys[(size_t)(p0 + j) * k + i] = lst[i];
      if (lane == 0) pair_cnt[p0 + j] = (uint32_t)size[u];
    }
  }
}

// ------------------------------------------------------ routing, tensor cores
// Posting-major batches under L2 with n_probe <= 64 and d <= 128 route on the
// tensor cores.  Queries and live centroids are centred on the mean m of (up
// to) 1024 live centroids, scaled per vector by a power of two (largest
// coordinate below 2^14) and split into FP16 halves x = hi + lo; k_route_tcm
// writes A = |q'|^2 + |c'|^2 - 2 q'.c' for every query x live centroid pair
// (q' = q - m, c' = c - m; q'.c' as qh.ch + qh.cl + ql.ch, FP32 accumulate).
// A is within
//     E(q) = 4e-4 (|q'|^2 + max_c |c'|^2)
// of the oracle's coordinate-order FP32 sum: the dropped lo.lo term and the
// split leave < 3 * 2^-22 |q'||c'|, the accumulation < 3 d * 2^-23 |q'||c'|,
// the norms, the centring and the oracle's own rounding < 3 (d + 4) * 2^-24
// (|q'|^2 + |c'|^2); for d <= 128 all together stay below a quarter of E.
// k_fr_select (a warp per query) then finds an upper bound U of the query's
// n_probe-th smallest A (the n_probe-th smallest of the four smallest values
// each lane saw), keeps every centroid with A <= U + 2 E(q) -- which holds
// for every centroid of the exact n_probe nearest, ties included -- computes
// their exact coordinate-order distances and takes the n_probe smallest
// (distance, slot) keys in ascending order: the probes, and the order, of the
// exact selection.  A query with more candidates than its list holds falls
// back to exact distances for every live centroid.
constexpr int kFrMeanRows = 1024;  // live centroids averaged for the centre
constexpr int kFrC = 64;           // centroids per staged tile (k_route_tcm)
constexpr int kFrTiles = 16;       // tiles per block of k_route_tcm
constexpr int kFrCap = 256;        // candidate list of a query (k_fr_select)
constexpr float kFrEps = 4e-4f;

__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }


// The power-of-two scale that brings a vector whose largest |coordinate| is
// mx below 2^14 (1 for a zero vector), and its inverse.
__device__ __forceinline__ float2 fr_scale(float mx) {
  if (!(mx > 0.0f)) return make_float2(1.0f, 1.0f);
  int e;
  frexpf(mx, &e);  // mx < 2^e
  return make_float2(ldexpf(1.0f, 14 - e), ldexpf(1.0f, e - 14));
}

// The centre: mean of the first min(live, 1024) live centroids (one block of
// 1024 threads, d <= 128); also clears the largest-norm word.
__global__ void __launch_bounds__(1024) k_fr_mean(const float *__restrict__ C, const uint32_t *__restrict__ cidx,
                                                  uint32_t d, uint32_t dpad, float *mu, uint32_t *maxcc_bits) {
  __shared__ float part[8][128];
  const uint32_t nl = __ldg(cidx), m = min(nl, (uint32_t)kFrMeanRows);
  const uint32_t i = threadIdx.x & 127, rg = threadIdx.x >> 7;
  float acc = 0.0f;
  if (i < d)
    for (uint32_t j = rg; j < m; j += 8) acc += __ldg(C + (size_t)__ldg(cidx + 1 + j) * dpad + i);
  part[rg][i] = acc;
  __syncthreads();
  if (rg == 0 && i < d) {
    float t = 0.0f;
    for (int r = 0; r < 8; ++r) t += part[r][i];
    mu[i] = m ? t / (float)m : 0.0f;
  }
  if (threadIdx.x == 0) *maxcc_bits = 0u;
}

// Per live centroid j (a warp each): c' = c - m, |c'|^2, FP16 hi / lo halves of
// c' s in rows of kd halves (zero padded past d), (|c'|^2, 1 / s), and the
// largest |c'|^2 (as float bits: norms are non-negative).
__global__ void __launch_bounds__(256) k_fr_centroids(const float *__restrict__ C, const uint32_t *__restrict__ cidx,
                                                      uint32_t d, uint32_t dpad, uint32_t kd,
                                                      const float *__restrict__ mu, __half *ch, __half *cl,
                                                      float2 *cinfo, uint32_t *maxcc_bits) {
  const uint32_t nl = __ldg(cidx);
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nl; j += nw) {
    const float *c = C + (size_t)__ldg(cidx + 1 + j) * dpad;
    float v[4], s2 = 0.0f, mx = 0.0f;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = lane + 32u * u;
      v[u] = i < d ? __fsub_rn(__ldg(c + i), __ldg(mu + i)) : 0.0f;
      s2 = fmaf(v[u], v[u], s2);
      mx = fmaxf(mx, fabsf(v[u]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s2 += __shfl_xor_sync(kFull, s2, o);
      mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    }
    const float2 sc = fr_scale(mx);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = lane + 32u * u;
      if (i < kd) {
        const float x = v[u] * sc.x;
        const __half h = __float2half_rn(x);
        ch[(size_t)j * kd + i] = h;
        cl[(size_t)j * kd + i] = __float2half_rn(x - __half2float(h));
      }
    }
    if (lane == 0) {
      cinfo[j] = make_float2(s2, sc.y);
      atomicMax(maxcc_bits, __float_as_uint(s2));
    }
  }
}

// seq_metric for L2 / squared L2 between 16-byte aligned rows (d % 4 == 0):
// the same coordinate-order arithmetic, four coordinates per load.
__device__ __forceinline__ float seq_l2_rows4(const float *q, const float *x, uint32_t d, int metric) {
  const float4 *q4 = reinterpret_cast<const float4 *>(q), *x4 = reinterpret_cast<const float4 *>(x);
  float acc = 0.0f;
#pragma unroll 4
  for (uint32_t i = 0; i < d / 4; ++i) {
    const float4 a = __ldg(q4 + i), b = __ldg(x4 + i);
    float t = __fsub_rn(a.x, b.x);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(a.y, b.y);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(a.z, b.z);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
    t = __fsub_rn(a.w, b.w);
    acc = __fadd_rn(acc, __fmul_rn(t, t));
  }
  return metric == DG_L2 ? __fsqrt_rn(acc) : acc;
}

// Per query q of a chunk (a warp each): q' = q - m, |q'|^2, FP16 hi / lo halves
// of q' s in rows of kd halves, and (|q'|^2, -2 / s, E(q), 0).
__global__ void __launch_bounds__(256) k_fr_queries(const float *__restrict__ Q, uint32_t nq, uint32_t qstride,
                                                    uint32_t d, uint32_t kd, const float *__restrict__ mu,
                                                    const uint32_t *__restrict__ maxcc_bits, __half *qh, __half *ql,
                                                    float4 *qinfo) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const float maxcc = __uint_as_float(__ldg(maxcc_bits));
  for (uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nq; q += nw) {
    float v[4], s2 = 0.0f, mx = 0.0f;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = lane + 32u * u;
      v[u] = i < d ? __fsub_rn(__ldg(Q + (size_t)q * qstride + i), __ldg(mu + i)) : 0.0f;
      s2 = fmaf(v[u], v[u], s2);
      mx = fmaxf(mx, fabsf(v[u]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s2 += __shfl_xor_sync(kFull, s2, o);
      mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
    }
    const float2 sc = fr_scale(mx);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint32_t i = lane + 32u * u;
      if (i < kd) {
        const float x = v[u] * sc.x;
        const __half h = __float2half_rn(x);
        qh[(size_t)q * kd + i] = h;
        ql[(size_t)q * kd + i] = __float2half_rn(x - __half2float(h));
      }
    }
    if (lane == 0) qinfo[q] = make_float4(s2, -2.0f * sc.y, __fmul_ru(kFrEps, __fadd_ru(s2, maxcc)), 0.0f);
  }
}

// A for 64 queries (4 warps x 16) x kFrTiles tiles of 64 live centroids per
// block, into D (rows ldd floats apart, ldd a multiple of 4).  Query
// fragments come straight from the hi / lo rows into registers; centroid
// tiles are staged in shared memory (double-buffered asynchronous copies) and
// read with ldmatrix.
template <int KS>
__global__ void __launch_bounds__(128) k_route_tcm(const __half *__restrict__ qh, const __half *__restrict__ ql,
                                                   const float4 *__restrict__ qinfo, uint32_t nq,
                                                   const __half *__restrict__ ch, const __half *__restrict__ cl,
                                                   const float2 *__restrict__ cinfo,
                                                   const uint32_t *__restrict__ cidx, float *__restrict__ D,
                                                   uint32_t ldd) {
  constexpr int KD = 16 * KS, RS = KD + 8;  // staged row stride (halves): conflict-free ldmatrix
  constexpr int CH = KD / 8;                // 16-byte chunks per row
  extern __shared__ __align__(16) uint8_t smem[];
  __half *tiles = reinterpret_cast<__half *>(smem);                         // [stage][hi, lo][kFrC][RS]
  float2 *tinfo = reinterpret_cast<float2 *>(smem + 2 * 2 * kFrC * RS * 2);  // [stage][kFrC]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const uint32_t nl = __ldg(cidx);
  const int t0 = blockIdx.y * kFrTiles;
  const int ntile = min(kFrTiles, (int)((nl + kFrC - 1) / kFrC) - t0);
  if (ntile <= 0) return;  // the whole block: past the live centroids
  const uint32_t qa = blockIdx.x * 64 + warp * 16 + g, qb = qa + 8;
  // A fragments: rows g, g + 8; k = 2t, 2t + 1 (+8) of each 16-dimension step
  uint32_t ah[KS][4], al[KS][4];
#pragma unroll
  for (int ks = 0; ks < KS; ++ks) {
    const uint32_t *ra = reinterpret_cast<const uint32_t *>(qh + (size_t)min(qa, nq - 1) * KD + 16 * ks + 2 * t);
    const uint32_t *rb = reinterpret_cast<const uint32_t *>(qh + (size_t)min(qb, nq - 1) * KD + 16 * ks + 2 * t);
    const uint32_t *la = reinterpret_cast<const uint32_t *>(ql + (size_t)min(qa, nq - 1) * KD + 16 * ks + 2 * t);
    const uint32_t *lb = reinterpret_cast<const uint32_t *>(ql + (size_t)min(qb, nq - 1) * KD + 16 * ks + 2 * t);
    ah[ks][0] = __ldg(ra);
    ah[ks][1] = __ldg(rb);
    ah[ks][2] = __ldg(ra + 4);
    ah[ks][3] = __ldg(rb + 4);
    al[ks][0] = __ldg(la);
    al[ks][1] = __ldg(lb);
    al[ks][2] = __ldg(la + 4);
    al[ks][3] = __ldg(lb + 4);
  }
  const float4 ia = __ldg(qinfo + min(qa, nq - 1)), ib = __ldg(qinfo + min(qb, nq - 1));
  auto stage = [&](int tt, int sb) {
    const uint32_t j0 = (uint32_t)(t0 + tt) * kFrC;
    for (int e = threadIdx.x; e < 2 * kFrC * CH; e += 128) {
      const int hl = e / (kFrC * CH), rem = e - hl * (kFrC * CH), r = rem / CH, c = rem - r * CH;
      const uint32_t j = j0 + r;
      const __half *src = (hl ? cl : ch) + (j < nl ? (size_t)j * KD + c * 8 : 0);
      cp_async16(tiles + ((size_t)(sb * 2 + hl) * kFrC + r) * RS + c * 8, src, j < nl ? 16u : 0u);
    }
    if (threadIdx.x < kFrC / 2) {
      const uint32_t j = j0 + 2 * threadIdx.x;
      cp_async16(tinfo + sb * kFrC + 2 * threadIdx.x, cinfo + (j < nl ? j : 0), j + 1 < nl ? 16u : (j < nl ? 8u : 0u));
    }
    cp_async_commit();
  };
  stage(0, 0);
  const uint32_t bo = 2u * (((lane >> 4) * 8 + (lane & 7)) * RS + ((lane >> 3) & 1) * 8);
  for (int tt = 0; tt < ntile; ++tt) {
    const int sb = tt & 1;
    if (tt + 1 < ntile) {
      stage(tt + 1, sb ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
    const uint32_t th_s = (uint32_t)__cvta_generic_to_shared(tiles + (size_t)(sb * 2) * kFrC * RS);
    const uint32_t tl_s = th_s + 2u * kFrC * RS;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        uint32_t bh[4], bl[4];
        const uint32_t off = bo + 2u * (16 * h * RS + 16 * ks);
        ldsm_x4(bh, th_s + off);
        ldsm_x4(bl, tl_s + off);
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          float(&c)[4] = acc[2 * h + o];
          mma_f16_16x8x16(c, ah[ks], bh[2 * o], bh[2 * o + 1]);
          mma_f16_16x8x16(c, ah[ks], bl[2 * o], bl[2 * o + 1]);
          mma_f16_16x8x16(c, al[ks], bh[2 * o], bh[2 * o + 1]);
        }
      }
    }
    // lane (g, t): queries qa, qb x centroids 2t, 2t + 1 of each 8-centroid n-tile
    const uint32_t j0 = (uint32_t)(t0 + tt) * kFrC;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int cc = 8 * nt + 2 * t;
      const uint32_t j = j0 + cc;
      const float2 c0 = tinfo[sb * kFrC + cc], c1 = tinfo[sb * kFrC + cc + 1];
      if (j < nl) {  // j even, ldd a multiple of 4: the pair is 8-byte aligned (column j + 1 may be padding)
        if (qa < nq)
          *reinterpret_cast<float2 *>(D + (size_t)qa * ldd + j) =
              make_float2(fmaf(ia.y * c0.y, acc[nt][0], __fadd_rn(ia.x, c0.x)),
                          fmaf(ia.y * c1.y, acc[nt][1], __fadd_rn(ia.x, c1.x)));
        if (qb < nq)
          *reinterpret_cast<float2 *>(D + (size_t)qb * ldd + j) =
              make_float2(fmaf(ib.y * c0.y, acc[nt][2], __fadd_rn(ib.x, c0.x)),
                          fmaf(ib.y * c1.y, acc[nt][3], __fadd_rn(ib.x, c1.x)));
      }
    }
    __syncthreads();  // every warp is done with this stage before it is refilled
  }
}

static size_t fr_tcm_smem(int ks) { return 2 * 2 * kFrC * (16 * (size_t)ks + 8) * 2 + 2 * kFrC * 8; }

// Probes of each query from its row of A (a warp per query, 4 per block):
// U = the n-th smallest of the four smallest values of every lane (U is at
// least the row's n-th smallest A), the live indices with A <= U + 2 E(q)
// into a list, their exact distances, the n smallest (distance, slot) keys,
// the probe_ratio cut of the query-major selection.
__global__ void __launch_bounds__(128) k_fr_select(const float *__restrict__ D, uint32_t ldd, uint32_t nq,
                                                   const float4 *__restrict__ qinfo, const float *__restrict__ Q,
                                                   uint32_t qstride, uint32_t d, const float *__restrict__ C,
                                                   uint32_t dpad, const uint32_t *__restrict__ cidx, int metric,
                                                   uint32_t nprobe, float probe_ratio, uint32_t *probe_out,
                                                   uint32_t *probe_cnt) {
  __shared__ uint32_t lists[4][kFrCap];
  __shared__ __align__(16) uint64_t keys[4][kFrCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t n = max(nprobe, 1u), nl = __ldg(cidx);
  const uint32_t *col = cidx + 1;
  uint32_t *lst = lists[warp];
  uint64_t *K = keys[warp];
  const float inf = __int_as_float(0x7f800000);
  for (uint32_t q = blockIdx.x * 4 + warp; q < nq; q += gridDim.x * 4) {
    const float *row = D + (size_t)q * ldd;
    const float4 *row4 = reinterpret_cast<const float4 *>(row);
    const uint32_t n4 = nl / 4;
    float bound = inf;
    if (nl > n) {
      // the four smallest values this lane sees
      float t0 = inf, t1 = inf, t2 = inf, t3 = inf;
      auto see = [&](float v) {
        if (v < t3) {
          t3 = v;
          if (t3 < t2) { const float x = t2; t2 = t3; t3 = x; }
          if (t2 < t1) { const float x = t1; t1 = t2; t2 = x; }
          if (t1 < t0) { const float x = t0; t0 = t1; t1 = x; }
        }
      };
      uint32_t i = lane;
      for (; i + 96 < n4; i += 128) {  // four loads in flight per lane
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = __ldg(row4 + i + 32 * u);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          see(v[u].x);
          see(v[u].y);
          see(v[u].z);
          see(v[u].w);
        }
      }
      for (; i < n4; i += 32) {
        const float4 v = __ldg(row4 + i);
        see(v.x);
        see(v.y);
        see(v.z);
        see(v.w);
      }
      if (4 * n4 + lane < nl) see(__ldg(row + 4 * n4 + lane));
      // U: the n-th smallest of the 128 kept values (ordered bits, bisection)
      const uint32_t u0 = ordered_bits(t0), u1 = ordered_bits(t1), u2 = ordered_bits(t2), u3 = ordered_bits(t3);
      uint32_t lo = 0, hi = 0xffffffffu;
      while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        const uint32_t c = __reduce_add_sync(kFull, (uint32_t)(u0 <= mid) + (u1 <= mid) + (u2 <= mid) + (u3 <= mid));
        if (c >= n) hi = mid;
        else lo = mid + 1;
      }
      bound = __fadd_ru(ordered_float(lo), 2.0f * __ldg(qinfo + q).z);
    }
    // the candidates: every live index with A <= bound (all of them when nl <= n)
    int m = 0;
    for (uint32_t i0 = 0; i0 < n4 + 1; i0 += 128) {  // four loads in flight per lane
      float4 v[4];
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        const uint32_t i = i0 + 32 * w + lane;
        v[w] = make_float4(inf, inf, inf, inf);
        if (i < n4) v[w] = __ldg(row4 + i);
        else if (i == n4) {
          if (4 * n4 < nl) v[w].x = __ldg(row + 4 * n4);
          if (4 * n4 + 1 < nl) v[w].y = __ldg(row + 4 * n4 + 1);
          if (4 * n4 + 2 < nl) v[w].z = __ldg(row + 4 * n4 + 2);
        }
      }
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        const uint32_t i = i0 + 32 * w + lane;
        const float vv[4] = {v[w].x, v[w].y, v[w].z, v[w].w};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const uint32_t j = 4 * i + u;
          const bool keep = j < nl && (vv[u] <= bound || nl <= n);
          const uint32_t km = __ballot_sync(kFull, keep);
          const int pos = m + __popc(km & lanemask_lt(lane));
          if (keep && pos < kFrCap) lst[pos] = j;
          m += __popc(km);
        }
      }
    }
    __syncwarp();
    const float *qg = Q + (size_t)q * qstride;
    int np;
    const uint64_t *sorted;
    if (m <= kFrCap) {
      constexpr int PL = kFrCap / 32;
      uint64_t kk[PL];
#pragma unroll
      for (int u = 0; u < PL; ++u) {
        const int x = lane + 32 * u;
        kk[u] = kKeyInvalid;
        if (x < m) {
          const uint32_t slot = __ldg(col + lst[x]);
          kk[u] = make_key(seq_l2_rows4(qg, C + (size_t)slot * dpad, d, metric), slot);
          K[x] = kk[u];
        }
      }
      __syncwarp();
      int rk[PL];
#pragma unroll
      for (int u = 0; u < PL; ++u) {
        rk[u] = 0;
        if (lane + 32 * u < m)
          for (int x = 0; x < m; ++x) rk[u] += K[x] < kk[u] ? 1 : 0;
      }
      __syncwarp();
      np = min((int)n, m);
#pragma unroll
      for (int u = 0; u < PL; ++u)
        if (lane + 32 * u < m && rk[u] < np) K[rk[u]] = kk[u];
      __syncwarp();
      sorted = K;
    } else {  // too many candidates: exact distances of every live centroid, a sorted list of n
      uint64_t *const P[2] = {K, K + 64};
      uint64_t *cst = K + 128;
      int cur = 0, size = 0;
      for (uint32_t j0 = 0; j0 < nl; j0 += 32) {
        const uint32_t j = j0 + lane;
        uint64_t key = kKeyInvalid;
        if (j < nl) {
          const uint32_t slot = __ldg(col + j);
          key = make_key(seq_l2_rows4(qg, C + (size_t)slot * dpad, d, metric), slot);
        }
        insert_batch(key, P, cur, size, (int)n, cst, lane);
      }
      np = size;
      sorted = P[cur];
    }
    // probe_ratio cut, as the query-major selection
    if (np > 0 && isfinite(probe_ratio)) {
      const float d0 = key_dist(sorted[0]);
      if (d0 >= 0.0f) {
        const float lim = __fmul_rn(d0, fmaxf(probe_ratio, 1.0f));
        int first_out = np;
        for (int i = lane; i < np; i += 32)
          if (key_dist(sorted[i]) > lim) first_out = min(first_out, i);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) first_out = min(first_out, __shfl_xor_sync(kFull, first_out, o));
        np = first_out;
      }
    }
    for (int i = lane; i < np; i += 32) probe_out[(size_t)q * nprobe + i] = key_id(sorted[i]);
    if (lane == 0) probe_cnt[q] = (uint32_t)np;
    __syncwarp();
  }
}

// The n nearest live postings of each row of an exact routing matrix (one
// warp per row), as (distance, slot) keys in ascending order: slots, distances.
__global__ void __launch_bounds__(128) k_route_topn(const float *__restrict__ D, uint32_t nv, uint32_t ldd,
                                                    const uint32_t *__restrict__ cidx, uint32_t n,
                                                    uint32_t *out_slots, float *out_d) {
  __shared__ __align__(16) uint64_t lists[4][2][64];
  __shared__ __align__(16) uint64_t cst[4][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t *const bufs[2] = {lists[warp][0], lists[warp][1]};
  const uint32_t nl = __ldg(cidx);
  for (uint32_t v = blockIdx.x * 4 + warp; v < nv; v += gridDim.x * 4) {
    int cur = 0, size = 0;
    for (uint32_t j0 = 0; j0 < nl; j0 += 32) {
      const uint32_t j = j0 + lane;
      const uint64_t key = j < nl ? make_key(D[(size_t)v * ldd + j], __ldg(cidx + 1 + j)) : kKeyInvalid;
      insert_batch(key, bufs, cur, size, (int)n, cst[warp], lane);
    }
    for (uint32_t i = lane; i < n; i += 32) {
      const bool ok = (int)i < size;
      out_slots[(size_t)v * n + i] = ok ? key_id(bufs[cur][i]) : DG_PAD;
      out_d[(size_t)v * n + i] = ok ? key_dist(bufs[cur][i]) : __int_as_float(0x7f800000);
    }
    __syncwarp();
  }
}

// Per query: the k best keys over its probed postings' pair lists.
__global__ void __launch_bounds__(128) k_pm_merge(const uint32_t *probe_cnt, const uint32_t *pos_of, uint32_t nq,
                                                  uint32_t nprobe, const uint64_t *pair_keys,
                                                  const uint32_t *pair_cnt, uint32_t k, uint64_t *out_ids,
                                                  float *out_d, uint32_t *out_cnt) {
  __shared__ __align__(16) uint64_t lists[4][2][kPmK];
  __shared__ __align__(16) uint64_t cst[4][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t *const bufs[2] = {lists[warp][0], lists[warp][1]};
  for (uint32_t q = blockIdx.x * 4 + warp; q < nq; q += gridDim.x * 4) {
    int cur = 0, size = 0;
    const uint32_t np = probe_cnt[q];
    for (uint32_t i = 0; i < np; ++i) {
      const uint32_t pos = pos_of[(size_t)q * nprobe + i];
      const uint32_t c = pair_cnt[pos];
      for (uint32_t j0 = 0; j0 < c; j0 += 32) {
        const uint32_t j = j0 + lane;
        insert_batch(j < c ? pair_keys[(size_t)pos * k + j] : kKeyInvalid, bufs, cur, size, (int)k, cst[warp], lane);
      }
    }
    const int count = min(size, (int)k);
    for (int i = lane; i < (int)k; i += 32) {
      out_ids[(size_t)q * k + i] = i < count ? (uint64_t)key_id(bufs[cur][i]) : DG_PAD64;
      out_d[(size_t)q * k + i] = i < count ? key_dist(bufs[cur][i]) : __int_as_float(0x7f800000);
    }
    if (lane == 0) out_cnt[q] = (uint32_t)count;
    __syncwarp();
  }
}

static size_t pm_smem(uint32_t d, uint32_t dpad, uint32_t k) {
  return ((size_t)kPmQ * dpad + (size_t)kPmT * (d + 4)) * 4 + (2 * kPmT + kPmQ) * 4 +
         (size_t)kPmQ * 2 * pm_kcap(k) * 8 + 8 * 32 * 8 + (size_t)(kPmQ + kPmT) * pm_ks(d) * 2;
}

// Posting-major scan of one chunk whose routing matrix is in ac.route: probes
// (the query-major kernel stops after selecting them), pairs grouped by
// posting, the scan, the per-query merge.
// Tensor-core routing state of one search (the live list fixed): the centre,
// the largest centred norm, per live centroid (|c'|^2, 1 / s) and FP16 halves,
// per query of a chunk (|q'|^2, -2 / s, E, 0) and FP16 halves, the A matrix.
struct FrPrep {
  float *mu;
  uint32_t *maxcc;
  float2 *cinfo;
  __half *ch, *cl, *qh, *ql;
  float4 *qinfo;
  float *D;
  uint32_t ldd;
  int ks;  // 16-dimension steps of the padded rows (2, 4, 6 or 8)
};

static DgStatus fr_prepare(DgSpfresh *s, const uint32_t *lidx, uint32_t chunk, cudaStream_t st, FrPrep *fp) {
  const int ks = s->d <= 32 ? 2 : s->d <= 64 ? 4 : s->d <= 96 ? 6 : 8;
  const size_t kd = 16 * (size_t)ks, nb = s->nblocks;
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t o_max = up(128 * 4), o_info = o_max + 256, o_h = o_info + up(nb * 8), o_l = o_h + up(nb * kd * 2),
               o_qi = o_l + up(nb * kd * 2), o_qh = o_qi + up((size_t)chunk * 16), o_ql = o_qh + up((size_t)chunk * kd * 2),
               total = o_ql + up((size_t)chunk * kd * 2);
  fp->ldd = (uint32_t)((nb + 3) & ~(size_t)3);
  DgStatus r;
  if ((r = buf_reserve(s->fr, total)) != DG_OK) return r;
  if ((r = buf_reserve(s->route, (size_t)chunk * fp->ldd * 4)) != DG_OK) return r;
  uint8_t *base = (uint8_t *)s->fr.p;
  fp->mu = (float *)base;
  fp->maxcc = (uint32_t *)(base + o_max);
  fp->cinfo = (float2 *)(base + o_info);
  fp->ch = (__half *)(base + o_h);
  fp->cl = (__half *)(base + o_l);
  fp->qinfo = (float4 *)(base + o_qi);
  fp->qh = (__half *)(base + o_qh);
  fp->ql = (__half *)(base + o_ql);
  fp->D = (float *)s->route.p;
  fp->ks = ks;
  k_fr_mean<<<1, 1024, 0, st>>>(s->centroids, lidx, s->d, s->dpad, fp->mu, fp->maxcc);
  k_fr_centroids<<<(unsigned)std::min<size_t>((nb + 7) / 8, 148 * 16), 256, 0, st>>>(
      s->centroids, lidx, s->d, s->dpad, (uint32_t)kd, fp->mu, fp->ch, fp->cl, fp->cinfo, fp->maxcc);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

template <int KS>
static DgStatus fr_matrix(const SpfArgs &ac, const FrPrep &fp, uint32_t nblocks, cudaStream_t st) {
  const size_t smem = fr_tcm_smem(KS);
  DG_CUDA(cudaFuncSetAttribute(k_route_tcm<KS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const uint32_t ntiles = (nblocks + kFrC - 1) / kFrC;
  dim3 grid((ac.nq + 63) / 64, std::max(1u, (ntiles + kFrTiles - 1) / kFrTiles));
  k_route_tcm<KS><<<grid, 128, smem, st>>>(fp.qh, fp.ql, fp.qinfo, ac.nq, fp.ch, fp.cl, fp.cinfo, ac.route_idx,
                                           fp.D, fp.ldd);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// The probes of a chunk's queries: query halves, the A matrix, the selection.
static DgStatus fr_route(const SpfArgs &ac, const FrPrep &fp, uint32_t nprobe, uint32_t nblocks, uint32_t *probe,
                         uint32_t *pcnt, cudaStream_t st) {
  const uint32_t kd = 16u * (uint32_t)fp.ks;
  k_fr_queries<<<(unsigned)std::min<size_t>(((size_t)ac.nq + 7) / 8, 148 * 16), 256, 0, st>>>(
      ac.Q, ac.nq, ac.d, ac.d, kd, fp.mu, fp.maxcc, fp.qh, fp.ql, fp.qinfo);
  DG_CUDA(cudaGetLastError());
  DgStatus r;
  switch (fp.ks) {
    case 2: r = fr_matrix<2>(ac, fp, nblocks, st); break;
    case 4: r = fr_matrix<4>(ac, fp, nblocks, st); break;
    case 6: r = fr_matrix<6>(ac, fp, nblocks, st); break;
    default: r = fr_matrix<8>(ac, fp, nblocks, st); break;
  }
  if (r != DG_OK) return r;
  k_fr_select<<<(unsigned)std::min<uint32_t>((ac.nq + 3) / 4, 148 * 16), 128, 0, st>>>(
      fp.D, fp.ldd, ac.nq, fp.qinfo, ac.Q, ac.d, ac.d, ac.centroids, ac.dpad, ac.route_idx, ac.metric, nprobe,
      ac.probe_ratio, probe, pcnt);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

static DgStatus pm_scan_chunk(DgSpfresh *s, const SpfArgs &ac, uint32_t nprobe, uint32_t k, uint32_t pcap,
                              uint32_t rcap, cudaStream_t st, const FrPrep *fp) {
  DgStatus r;
  const uint32_t qn = ac.nq, nb = s->nblocks;
  const size_t npairs = (size_t)qn * nprobe;
  const size_t nitems = npairs / kPmQ + nb + 1;
  if ((r = buf_reserve(s->probe, npairs * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->probe_cnt, (size_t)qn * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->pcount, ((size_t)nb + 1) * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->pstart, ((size_t)nb + 1) * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->pfill, ((size_t)nb + 1) * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->istart, ((size_t)nb + 1) * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->pair_q, npairs * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->pos_of, npairs * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->items, nitems * 16)) != DG_OK) return r;
  if ((r = buf_reserve(s->pair_keys, npairs * k * 8)) != DG_OK) return r;
  if ((r = buf_reserve(s->pair_cnt, npairs * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->misc, 16)) != DG_OK) return r;
  if ((r = buf_reserve(s->qthr, (size_t)qn * 4)) != DG_OK) return r;
  uint32_t *probe = (uint32_t *)s->probe.p, *pcnt = (uint32_t *)s->probe_cnt.p;
  uint32_t *pcount = (uint32_t *)s->pcount.p, *pstart = (uint32_t *)s->pstart.p, *pfill = (uint32_t *)s->pfill.p;
  uint32_t *istart = (uint32_t *)s->istart.p, *counter = (uint32_t *)s->misc.p;
  if (nprobe > 64) {
    // wide probes: radix select (a sorted list of nprobe keys costs more)
    k_pm_select<<<(unsigned)std::min<uint32_t>((qn + 3) / 4, 148 * 16), 128, 0, st>>>(
        ac.route, ac.route_idx, qn, nb, nprobe, ac.probe_ratio, probe, pcnt);
    DG_CUDA(cudaGetLastError());
  } else if (fp) {
    // tensor-core routing: the A matrix, then exact distances near the cut
    if ((r = fr_route(ac, *fp, nprobe, nb, probe, pcnt, st)) != DG_OK) return r;
  } else {
    // the query-major kernel's selection, stopped before its scan
    SpfArgs ap = ac;
    ap.probe_out = probe;
    ap.probe_cnt = pcnt;
    DG_CUDA(cudaMemsetAsync(ap.counter, 0, 4, st));
    if ((r = spf_launch<SPF_RAW, MET_L2>(ap, pcap, rcap, st)) != DG_OK) return r;
  }
  DG_CUDA(cudaMemsetAsync(pcount, 0, ((size_t)nb + 1) * 4, st));
  DG_CUDA(cudaMemsetAsync(pfill, 0, ((size_t)nb + 1) * 4, st));
  DG_CUDA(cudaMemsetAsync(counter, 0, 4, st));
  const unsigned gp = (unsigned)std::min<size_t>((npairs + 255) / 256, 148 * 16);
  k_pm_count<<<gp, 256, 0, st>>>(probe, pcnt, qn, nprobe, pcount);
  k_pm_scan<<<1, 1024, 0, st>>>(pcount, nb, pstart, istart);
  k_pm_scatter<<<gp, 256, 0, st>>>(probe, pcnt, qn, nprobe, pstart, pfill, (uint32_t *)s->pair_q.p,
                                   (uint32_t *)s->pos_of.p);
  k_pm_items<<<(nb + 255) / 256, 256, 0, st>>>(pcount, pstart, istart, nb, (uint4 *)s->items.p);
  DG_CUDA(cudaGetLastError());
  const size_t smem = pm_smem(s->d, s->dpad, k);
  DG_CUDA(cudaFuncSetAttribute(k_pm_scan_postings, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0, sms = 0;
  DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pm_scan_postings, 256, smem));
  DG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
  if (per_sm < 1) return fail(DG_ENOTSUP, "posting-major scan does not fit on an SM");
  uint32_t *qthr = (uint32_t *)s->qthr.p;
  const size_t bsmem = (size_t)4 * s->cap * 4;
  if (bsmem <= 160 * 1024) {
    DG_CUDA(cudaFuncSetAttribute(k_pm_bound, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsmem));
    k_pm_bound<<<(unsigned)std::min<uint32_t>((qn + 3) / 4, 148 * 16), 128, bsmem, st>>>(ac, probe, pcnt, nprobe,
                                                                                           k, qthr);
  } else {
    DG_CUDA(cudaMemsetAsync(qthr, 0xff, (size_t)qn * 4, st));  // no bound: every entry goes to its pair list
  }
  k_pm_scan_postings<<<per_sm * sms, 256, smem, st>>>(ac, (const uint4 *)s->items.p, istart + nb, counter,
                                                      (const uint32_t *)s->pair_q.p, (uint64_t *)s->pair_keys.p,
                                                      (uint32_t *)s->pair_cnt.p, k, qthr);
  k_pm_merge<<<(unsigned)std::min<uint32_t>((qn + 3) / 4, 148 * 16), 128, 0, st>>>(
      pcnt, (const uint32_t *)s->pos_of.p, qn, nprobe, (const uint64_t *)s->pair_keys.p,
      (const uint32_t *)s->pair_cnt.p, k, ac.out_ids, ac.out_d, ac.out_cnt);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

template <int KIND>
static DgStatus spf_launch_met(const SpfArgs &a, int met, uint32_t pcap, uint32_t rcap, cudaStream_t st) {
  if (met == MET_L2) return spf_launch<KIND, MET_L2>(a, pcap, rcap, st);
  if (met == MET_DOT) return spf_launch<KIND, MET_DOT>(a, pcap, rcap, st);
  return spf_launch<KIND, MET_COS>(a, pcap, rcap, st);
}

static DgStatus spf_alloc(DgSpfresh *s, void **p, size_t bytes) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  s->allocs.push_back(q);
  *p = q;
  return DG_OK;
}

}  // namespace dg

using namespace dg;

extern "C" {

DgStatus dg_spfresh_destroy(DgSpfresh *s) {
  if (!s) return DG_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->searched) {
    cudaEventSynchronize(s->searched);
    cudaEventDestroy(s->searched);
  }
  for (void *p : s->allocs) cudaFree(p);
  for (DgIndex::Buf *b : {&s->q, &s->oids, &s->od, &s->ocnt, &s->route, &s->live_idx, &s->fr, &s->probe, &s->probe_cnt,
                          &s->pcount, &s->pstart, &s->pfill, &s->istart, &s->pair_q, &s->pos_of, &s->items,
                          &s->pair_keys, &s->pair_cnt, &s->misc, &s->qthr})
    if (b->p) cudaFree(b->p);
  if (s->counter) cudaFree(s->counter);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DG_OK;
}

DgStatus dg_spfresh_create(const DgSpfreshDesc *desc, DgSpfresh **out) {
  if (!desc || !out) return fail(DG_EINVAL, "null argument");
  *out = nullptr;
  if (desc->dim == 0 || desc->num_blocks == 0 || desc->block_cap == 0)
    return fail(DG_EINVAL, "SPFresh needs dim, num_blocks and block_cap >= 1");
  if (desc->id_capacity >= (1ull << 31)) return fail(DG_EINVAL, "SPFresh ids must stay below 2^31");
  if ((uint64_t)desc->num_blocks * desc->block_cap >= (1ull << 32)) return fail(DG_EINVAL, "too many posting slots");
  if (desc->metric < DG_L2SQ || desc->metric > DG_DOT) return fail(DG_EINVAL, "unknown metric");
  if (!desc->centroids || !desc->block_live || !desc->block_len || !desc->entry_ids || !desc->raw)
    return fail(DG_EINVAL, "centroids, block arrays, entry ids and raw vectors are required");
  const uint32_t d = desc->dim, dpad = dpad_of(d);
  uint32_t code_size = 0;
  switch (desc->quantizer) {
    case DG_Q_NONE: code_size = d * 4; break;
    case DG_Q_F16: code_size = d * 2; break;
    case DG_Q_INT8: code_size = d; break;
    case DG_Q_PQ:
      if (!desc->pq_codebooks || desc->pq_M == 0 || d % desc->pq_M || desc->pq_K == 0 || desc->pq_K > 256)
        return fail(DG_EINVAL, "bad PQ parameters");
      code_size = desc->pq_M;
      break;
    case DG_Q_RABITQ: {
      uint32_t want = 1;
      while (want < std::max(d, 64u)) want <<= 1;
      if (desc->rq_padded != want || !desc->rq_signs) return fail(DG_EINVAL, "bad RaBitQ parameters");
      code_size = want / 8 + 8;
      break;
    }
    default: return fail(DG_EINVAL, "unknown quantizer");
  }
  if (desc->code_size != code_size)
    return fail(DG_EINVAL, "code_size must be " + std::to_string(code_size) + " for this quantizer and dimension");
  if (!desc->entry_codes) return fail(DG_EINVAL, "entry codes are required");
  DG_CUDA(cudaSetDevice(desc->device));
  DgSpfresh *s = new (std::nothrow) DgSpfresh();
  if (!s) return fail(DG_ENOMEM, "host allocation failed");
  auto bail = [&](DgStatus st) {
    dg_spfresh_destroy(s);
    return st;
  };
  s->device = desc->device;
  s->d = d;
  s->dpad = dpad;
  s->nblocks = desc->num_blocks;
  s->cap = desc->block_cap;
  s->metric = desc->metric;
  s->quant = desc->quantizer;
  s->code_size = code_size;
  // raw codes are rows of the padded dimension so they share the FP32 gather
  s->code_stride = desc->quantizer == DG_Q_NONE ? dpad * 4
                   : desc->quantizer == DG_Q_F16 ? dpad * 2
                   : desc->quantizer == DG_Q_INT8 ? dpad
                                                  : ((code_size + 15u) & ~15u);
  s->id_cap = desc->id_capacity;
  s->pq_M = desc->pq_M;
  s->pq_K = desc->pq_K;
  s->i8_scale = desc->int8_scale;
  s->i8_offset = desc->int8_offset;
  s->rq_padded = desc->rq_padded;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(DG_EDEVICE, "stream creation failed"));
  if (cudaEventCreateWithFlags(&s->searched, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(DG_EDEVICE, "event creation failed"));
  DgStatus st;
  const size_t nb = s->nblocks, slots = nb * s->cap;
  if ((st = spf_alloc(s, (void **)&s->centroids, nb * dpad * 4)) != DG_OK) return bail(st);
  if ((st = spf_alloc(s, (void **)&s->live, nb)) != DG_OK) return bail(st);
  if ((st = spf_alloc(s, (void **)&s->len, nb * 4)) != DG_OK) return bail(st);
  if ((st = spf_alloc(s, (void **)&s->ids, slots * 4)) != DG_OK) return bail(st);
  if ((st = spf_alloc(s, (void **)&s->codes, slots * s->code_stride)) != DG_OK) return bail(st);
  if ((st = spf_alloc(s, (void **)&s->deleted, ((s->id_cap + 31) / 32 + 1) * 4)) != DG_OK) return bail(st);
  if ((st = spf_alloc(s, (void **)&s->raw, std::max<uint64_t>(s->id_cap, 1) * dpad * 4)) != DG_OK) return bail(st);
  if (cudaMalloc(&s->counter, 4) != cudaSuccess) return bail(fail(DG_ENOMEM, "counter allocation"));
  cudaStream_t ss = s->stream;
  if ((st = upload_rows_f32(desc->centroids, nb, d, dpad, s->centroids, ss)) != DG_OK) return bail(st);
  DG_CUDA(cudaMemcpyAsync(s->live, desc->block_live, nb, cudaMemcpyHostToDevice, ss));
  DG_CUDA(cudaMemcpyAsync(s->len, desc->block_len, nb * 4, cudaMemcpyHostToDevice, ss));
  {
    std::vector<uint32_t> ids32(slots);
    for (size_t i = 0; i < slots; ++i) {
      const uint64_t v = desc->entry_ids[i];
      if (v != DG_PAD64 && v >= s->id_cap) return bail(fail(DG_EINVAL, "entry id beyond id_capacity"));
      ids32[i] = v == DG_PAD64 ? 0u : (uint32_t)v;
    }
    for (size_t b = 0; b < nb; ++b)
      if (desc->block_len[b] > s->cap) return bail(fail(DG_EINVAL, "block_len above block_cap"));
    DG_CUDA(cudaMemcpyAsync(s->ids, ids32.data(), slots * 4, cudaMemcpyHostToDevice, ss));
    DG_CUDA(cudaStreamSynchronize(ss));
  }
  DG_CUDA(cudaMemsetAsync(s->codes, 0, slots * s->code_stride, ss));
  DG_CUDA(cudaMemcpy2DAsync(s->codes, s->code_stride, desc->entry_codes, code_size, code_size, slots,
                            cudaMemcpyHostToDevice, ss));
  DG_CUDA(cudaMemsetAsync(s->deleted, 0, ((s->id_cap + 31) / 32 + 1) * 4, ss));
  if (desc->deleted) {
    std::vector<uint32_t> bm((s->id_cap + 31) / 32 + 1, 0u);
    for (uint64_t i = 0; i < s->id_cap; ++i)
      if (desc->deleted[i]) bm[i >> 5] |= 1u << (i & 31);
    DG_CUDA(cudaMemcpyAsync(s->deleted, bm.data(), bm.size() * 4, cudaMemcpyHostToDevice, ss));
    DG_CUDA(cudaStreamSynchronize(ss));
  }
  if ((st = upload_rows_f32(desc->raw, desc->num_raw, d, dpad, s->raw, ss)) != DG_OK) return bail(st);
  if (desc->quantizer == DG_Q_PQ) {
    const size_t cbb = (size_t)s->pq_M * s->pq_K * (d / s->pq_M) * 4;
    if ((st = spf_alloc(s, (void **)&s->pq_cb, cbb)) != DG_OK) return bail(st);
    DG_CUDA(cudaMemcpyAsync(s->pq_cb, desc->pq_codebooks, cbb, cudaMemcpyHostToDevice, ss));
  }
  if (desc->quantizer == DG_Q_RABITQ) {
    if ((st = spf_alloc(s, (void **)&s->rq_signs, 3ull * s->rq_padded * 4)) != DG_OK) return bail(st);
    DG_CUDA(cudaMemcpyAsync(s->rq_signs, desc->rq_signs, 3ull * s->rq_padded * 4, cudaMemcpyHostToDevice, ss));
  }
  if (cudaStreamSynchronize(ss) != cudaSuccess) return bail(fail(DG_EDEVICE, "upload failed"));
  *out = s;
  return DG_OK;
}

DgStatus dg_spfresh_update_blocks(DgSpfresh *s, const uint32_t *blocks, uint32_t nupd, const float *centroids,
                                  const uint8_t *live, const uint32_t *lens, const uint64_t *entry_ids,
                                  const uint8_t *entry_codes) {
  if (!s || (nupd && (!blocks || !centroids || !live || !lens || !entry_ids || !entry_codes)))
    return fail(DG_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  DG_CUDA(cudaSetDevice(s->device));
  cudaStream_t ss = s->stream;
  DG_CUDA(cudaStreamWaitEvent(ss, s->searched, 0));
  std::vector<uint32_t> ids32(s->cap);
  for (uint32_t u = 0; u < nupd; ++u) {
    const uint32_t b = blocks[u];
    if (b >= s->nblocks) return fail(DG_EINVAL, "block index out of range");
    if (lens[u] > s->cap) return fail(DG_EINVAL, "block_len above block_cap");
    for (uint32_t i = 0; i < s->cap; ++i) {
      const uint64_t v = entry_ids[(size_t)u * s->cap + i];
      if (i < lens[u] && v >= s->id_cap) return fail(DG_EINVAL, "entry id beyond id_capacity");
      ids32[i] = i < lens[u] ? (uint32_t)v : 0u;
    }
    DG_CUDA(cudaMemcpyAsync(s->ids + (size_t)b * s->cap, ids32.data(), s->cap * 4, cudaMemcpyHostToDevice, ss));
    DgStatus st = upload_rows_f32(centroids + (size_t)u * s->d, 1, s->d, s->dpad, s->centroids + (size_t)b * s->dpad, ss);
    if (st != DG_OK) return st;
    DG_CUDA(cudaMemcpyAsync(s->live + b, live + u, 1, cudaMemcpyHostToDevice, ss));
    DG_CUDA(cudaMemcpyAsync(s->len + b, lens + u, 4, cudaMemcpyHostToDevice, ss));
    uint8_t *dst = s->codes + (size_t)b * s->cap * s->code_stride;
    DG_CUDA(cudaMemsetAsync(dst, 0, (size_t)s->cap * s->code_stride, ss));
    DG_CUDA(cudaMemcpy2DAsync(dst, s->code_stride, entry_codes + (size_t)u * s->cap * s->code_size, s->code_size,
                              s->code_size, s->cap, cudaMemcpyHostToDevice, ss));
    DG_CUDA(cudaStreamSynchronize(ss));  // ids32 is reused for the next block
  }
  return DG_OK;
}

DgStatus dg_spfresh_set_centroids(DgSpfresh *s, const uint32_t *blocks, uint32_t nupd, const float *centroids,
                                  const uint8_t *live) {
  if (!s || (nupd && (!blocks || !centroids || !live))) return fail(DG_EINVAL, "null argument");
  for (uint32_t u = 0; u < nupd; ++u)
    if (blocks[u] >= s->nblocks) return fail(DG_EINVAL, "block index out of range");
  std::lock_guard<std::mutex> lk(s->mu);
  DG_CUDA(cudaSetDevice(s->device));
  cudaStream_t ss = s->stream;
  DG_CUDA(cudaStreamWaitEvent(ss, s->searched, 0));
  for (uint32_t u = 0; u < nupd; ++u) {
    const uint32_t b = blocks[u];
    DgStatus st = upload_rows_f32(centroids + (size_t)u * s->d, 1, s->d, s->dpad, s->centroids + (size_t)b * s->dpad, ss);
    if (st != DG_OK) return st;
    DG_CUDA(cudaMemcpyAsync(s->live + b, live + u, 1, cudaMemcpyHostToDevice, ss));
  }
  DG_CUDA(cudaStreamSynchronize(ss));  // the host arrays may go once this returns
  return DG_OK;
}

DgStatus dg_spfresh_nearest(DgSpfresh *s, const float *vectors, uint32_t nv, uint32_t n, uint32_t *out_slots,
                            float *out_dists) {
  if (!s || (nv && (!vectors || !out_slots || !out_dists))) return fail(DG_EINVAL, "null argument");
  if (n == 0 || n > 64) return fail(DG_EINVAL, "n must be in [1, 64]");
  if (nv == 0) return DG_OK;
  std::lock_guard<std::mutex> lk(s->mu);
  DG_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  DG_CUDA(cudaStreamWaitEvent(st, s->searched, 0));  // shares the search's scratch
  DgStatus r;
  const uint32_t chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nv, (1ull << 28) / s->nblocks));
  if ((r = buf_reserve(s->q, (size_t)nv * s->d * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->route, (size_t)chunk * s->nblocks * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->live_idx, ((size_t)s->nblocks + 1) * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->oids, (size_t)nv * n * 4)) != DG_OK) return r;
  if ((r = buf_reserve(s->od, (size_t)nv * n * 4)) != DG_OK) return r;
  DG_CUDA(cudaMemcpyAsync(s->q.p, vectors, (size_t)nv * s->d * 4, cudaMemcpyHostToDevice, st));
  uint32_t *lidx = (uint32_t *)s->live_idx.p;
  DG_CUDA(cudaMemsetAsync(lidx, 0, 4, st));
  k_live_idx<<<(s->nblocks + 255) / 256, 256, 0, st>>>(s->live, s->nblocks, lidx);
  for (uint32_t v0 = 0; v0 < nv; v0 += chunk) {
    const uint32_t vn = std::min(chunk, nv - v0);
    const float *Qc = (const float *)s->q.p + (size_t)v0 * s->d;
    dim3 grid((s->nblocks + kRT - 1) / kRT, (vn + kRT - 1) / kRT);
    k_route<<<grid, 256, 0, st>>>(Qc, vn, s->d, s->centroids, lidx, s->d, s->dpad, s->metric, (float *)s->route.p,
                                  s->nblocks);
    k_route_topn<<<(unsigned)std::min<uint32_t>((vn + 3) / 4, 148 * 16), 128, 0, st>>>(
        (const float *)s->route.p, vn, s->nblocks, lidx, n, (uint32_t *)s->oids.p + (size_t)v0 * n,
        (float *)s->od.p + (size_t)v0 * n);
  }
  DG_CUDA(cudaGetLastError());
  DG_CUDA(cudaMemcpyAsync(out_slots, s->oids.p, (size_t)nv * n * 4, cudaMemcpyDeviceToHost, st));
  DG_CUDA(cudaMemcpyAsync(out_dists, s->od.p, (size_t)nv * n * 4, cudaMemcpyDeviceToHost, st));
  DG_CUDA(cudaEventRecord(s->searched, st));
  DG_CUDA(cudaStreamSynchronize(st));
  return DG_OK;
}

DgStatus dg_spfresh_put_raw(DgSpfresh *s, uint64_t first_id, const float *vectors, uint64_t n) {
  if (!s || (n && !vectors)) return fail(DG_EINVAL, "null argument");
  if (first_id + n > s->id_cap) return fail(DG_EINVAL, "raw rows beyond id_capacity");
  std::lock_guard<std::mutex> lk(s->mu);
  DG_CUDA(cudaSetDevice(s->device));
  DG_CUDA(cudaStreamWaitEvent(s->stream, s->searched, 0));
  DgStatus st = upload_rows_f32(vectors, n, s->d, s->dpad, s->raw + first_id * s->dpad, s->stream);
  if (st != DG_OK) return st;
  DG_CUDA(cudaStreamSynchronize(s->stream));
  return DG_OK;
}

DgStatus dg_spfresh_set_deleted(DgSpfresh *s, const uint64_t *ids, uint64_t n, int32_t deleted) {
  if (!s || (n && !ids)) return fail(DG_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  DG_CUDA(cudaSetDevice(s->device));
  DG_CUDA(cudaStreamWaitEvent(s->stream, s->searched, 0));
  const size_t words = (s->id_cap + 31) / 32 + 1;
  std::vector<uint32_t> bm(words);
  DG_CUDA(cudaMemcpyAsync(bm.data(), s->deleted, words * 4, cudaMemcpyDeviceToHost, s->stream));
  DG_CUDA(cudaStreamSynchronize(s->stream));
  for (uint64_t i = 0; i < n; ++i) {
    if (ids[i] >= s->id_cap) return fail(DG_EINVAL, "id beyond id_capacity");
    if (deleted) bm[ids[i] >> 5] |= 1u << (ids[i] & 31);
    else bm[ids[i] >> 5] &= ~(1u << (ids[i] & 31));
  }
  DG_CUDA(cudaMemcpyAsync(s->deleted, bm.data(), words * 4, cudaMemcpyHostToDevice, s->stream));
  DG_CUDA(cudaStreamSynchronize(s->stream));
  return DG_OK;
}

DgStatus dg_spfresh_search_batch(DgSpfresh *s, const DgSpfreshParams *p, const float *queries, uint32_t nq,
                                 uint64_t *out_ids, float *out_dists, uint32_t *out_counts) {
  if (!s || !p) return fail(DG_EINVAL, "null argument");
  if (nq == 0) return DG_OK;
  if (!queries || !out_ids || !out_dists || !out_counts) return fail(DG_EINVAL, "null buffer");
  if (p->k == 0) return fail(DG_EINVAL, "k must be >= 1");
  const uint32_t nprobe = std::max(p->nprobe, 1u);
  const bool rq = s->quant == DG_Q_RABITQ && (s->metric == DG_L2 || s->metric == DG_L2SQ);
  const bool rerank = s->quant != DG_Q_NONE && !rq && p->rerank_size > 0;
  const uint32_t want = rerank ? std::max(p->k, p->rerank_size) : p->k;
  auto cap_of = [](uint32_t x) -> uint32_t { return x <= 64 ? 64 : x <= 256 ? 256 : x <= 1024 ? 1024 : 0; };
  const uint32_t pcap = cap_of(nprobe), rcap = cap_of(want);
  if (!pcap) return fail(DG_ENOTSUP, "n_probe above 1024");
  if (!rcap) return fail(DG_ENOTSUP, "k / rerank_size above 1024");
  const bool devptr = (p->flags & DG_FLAG_DEVICE_PTRS) != 0;
  std::lock_guard<std::mutex> lk(s->mu);
  DG_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = (p->flags & DG_FLAG_STREAM) || p->stream ? (cudaStream_t)p->stream : s->stream;
  DG_CUDA(cudaStreamWaitEvent(st, s->searched, 0));  // the previous search's scratch is free again
  SpfArgs a{};
  a.d = s->d;
  a.dpad = s->dpad;
  a.nblocks = s->nblocks;
  a.cap = s->cap;
  a.metric = s->metric;
  a.centroids = s->centroids;
  a.live = s->live;
  a.len = s->len;
  a.ids = s->ids;
  a.codes = s->codes;
  a.code_stride = s->code_stride;
  a.deleted = s->deleted;
  a.raw = s->raw;
  a.pq_M = s->pq_M;
  a.pq_K = s->pq_K;
  a.pq_ds = s->pq_M ? s->d / s->pq_M : 0;
  a.pq_cb = s->pq_cb;
  a.i8_scale = s->i8_scale;
  a.i8_offset = s->i8_offset;
  a.rq_padded = s->rq_padded;
  a.rq_signs = s->rq_signs;
  a.nq = nq;
  a.k = p->k;
  a.nprobe = nprobe;
  a.rerank = rerank ? p->rerank_size : 0;
  a.probe_ratio = p->probe_ratio;
  a.counter = s->counter;
  DgStatus r;
  const size_t kq = (size_t)nq * p->k;
  if (devptr) {
    a.Q = queries;
    a.out_ids = out_ids;
    a.out_d = out_dists;
    a.out_cnt = out_counts;
  } else {
    if ((r = buf_reserve(s->q, (size_t)nq * s->d * 4)) != DG_OK) return r;
    if ((r = buf_reserve(s->oids, kq * 8)) != DG_OK) return r;
    if ((r = buf_reserve(s->od, kq * 4)) != DG_OK) return r;
    if ((r = buf_reserve(s->ocnt, (size_t)nq * 4)) != DG_OK) return r;
    DG_CUDA(cudaMemcpyAsync(s->q.p, queries, (size_t)nq * s->d * 4, cudaMemcpyHostToDevice, st));
    a.Q = (const float *)s->q.p;
    a.out_ids = (uint64_t *)s->oids.p;
    a.out_d = (float *)s->od.p;
    a.out_cnt = (uint32_t *)s->ocnt.p;
  }
  const int met = s->metric == DG_DOT ? MET_DOT : s->metric == DG_COSINE ? MET_COS : MET_L2;
  auto scan = [&](const SpfArgs &aa) -> DgStatus {
    DG_CUDA(cudaMemsetAsync(s->counter, 0, 4, st));
    switch (s->quant) {
      case DG_Q_NONE: return spf_launch_met<SPF_RAW>(aa, met, pcap, rcap, st);
      case DG_Q_PQ: return spf_launch_met<SPF_PQ>(aa, met, pcap, rcap, st);
      case DG_Q_INT8: return spf_launch_met<SPF_INT8>(aa, met, pcap, rcap, st);
      case DG_Q_F16: return spf_launch_met<SPF_F16>(aa, met, pcap, rcap, st);
      default: return spf_launch_met<SPF_RABITQ>(aa, met, pcap, rcap, st);
    }
  };
  // raw f32 postings under L2 in batches that probe each posting from about 16
  // queries or more: the posting-major scan (each probed posting read once per
  // chunk instead of once per probing query); sparser batches stay query-major
  const bool posting_major = s->nblocks >= 512 && s->quant == DG_Q_NONE &&
                             (s->metric == DG_L2 || s->metric == DG_L2SQ) && p->k <= (uint32_t)kPmK && nq >= 256 &&
                             (uint64_t)nq * nprobe >= 16ull * s->nblocks && s->nblocks < (1u << 22) && s->d % 4 == 0 &&
                             pm_smem(s->d, s->dpad, p->k) <= 200 * 1024;
  // DG_SPF_EXACT_ROUTE=1 routes with the exact FP32 kernel only (an A/B knob)
  static const bool exact_only = std::getenv("DG_SPF_EXACT_ROUTE") && atoi(std::getenv("DG_SPF_EXACT_ROUTE"));
  // batches of >= 256 queries under L2 with n_probe <= 64 and d <= 128 route on
  // the tensor cores (exact distances only near each query's cut)
  const bool tc_route = s->nblocks >= 512 && (s->metric == DG_L2 || s->metric == DG_L2SQ) && nq >= 256 &&
                        nprobe <= 64 && s->d <= 128 && s->d % 4 == 0 && ((uintptr_t)a.Q & 15) == 0 && !exact_only;
  if (s->nblocks >= 512) {
    // many postings: route all queries of a chunk in one tiled kernel (the
    // matrix of a chunk stays below 2 GiB), then scan the chunk
    const uint32_t chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nq, (1ull << 29) / s->nblocks));
    if (!tc_route && (r = buf_reserve(s->route, (size_t)chunk * s->nblocks * 4)) != DG_OK) return r;
    if ((r = buf_reserve(s->live_idx, ((size_t)s->nblocks + 1) * 4)) != DG_OK) return r;
    uint32_t *lidx = (uint32_t *)s->live_idx.p;
    DG_CUDA(cudaMemsetAsync(lidx, 0, 4, st));
    k_live_idx<<<(s->nblocks + 255) / 256, 256, 0, st>>>(s->live, s->nblocks, lidx);
    DG_CUDA(cudaGetLastError());
    FrPrep fp{};
    if (tc_route && (r = fr_prepare(s, lidx, chunk, st, &fp)) != DG_OK) return r;
    for (uint32_t q0 = 0; q0 < nq; q0 += chunk) {
      const uint32_t qn = std::min(chunk, nq - q0);
      SpfArgs ac = a;
      ac.Q = a.Q + (size_t)q0 * s->d;
      ac.nq = qn;
      ac.out_ids = a.out_ids + (size_t)q0 * p->k;
      ac.out_d = a.out_d + (size_t)q0 * p->k;
      ac.out_cnt = a.out_cnt + q0;
      ac.route = tc_route ? nullptr : (const float *)s->route.p;
      ac.route_idx = lidx;
      if (!tc_route) {
        dim3 grid((s->nblocks + kRT - 1) / kRT, (qn + kRT - 1) / kRT);
        k_route<<<grid, 256, 0, st>>>(ac.Q, qn, s->d, s->centroids, lidx, s->d, s->dpad, s->metric,
                                      (float *)s->route.p, s->nblocks);
        DG_CUDA(cudaGetLastError());
      }
      if (posting_major) {
        if ((r = pm_scan_chunk(s, ac, nprobe, p->k, pcap, rcap, st, tc_route ? &fp : nullptr)) != DG_OK) return r;
      } else if (tc_route) {  // probes first, then the query-major scan of them
        if ((r = buf_reserve(s->probe, (size_t)qn * nprobe * 4)) != DG_OK) return r;
        if ((r = buf_reserve(s->probe_cnt, (size_t)qn * 4)) != DG_OK) return r;
        if ((r = fr_route(ac, fp, nprobe, s->nblocks, (uint32_t *)s->probe.p, (uint32_t *)s->probe_cnt.p, st)) != DG_OK)
          return r;
        ac.probe_in = (const uint32_t *)s->probe.p;
        ac.probe_in_cnt = (const uint32_t *)s->probe_cnt.p;
        if ((r = scan(ac)) != DG_OK) return r;
      } else if ((r = scan(ac)) != DG_OK) {
        return r;
      }
    }
  } else if ((r = scan(a)) != DG_OK) {
    return r;
  }
  if (!devptr) {
    DG_CUDA(cudaMemcpyAsync(out_ids, a.out_ids, kq * 8, cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaMemcpyAsync(out_dists, a.out_d, kq * 4, cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaMemcpyAsync(out_counts, a.out_cnt, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
  }
  DG_CUDA(cudaEventRecord(s->searched, st));
  if (!devptr) DG_CUDA(cudaStreamSynchronize(st));
  return DG_OK;
}

}  // extern "C"
