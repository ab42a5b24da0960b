// dg_search_kernel.cuh -- the persistent beam-search kernel template.
#pragma once
#include "dg_search.cuh"

namespace dg {

// |q|^2 for the cosine metric.  Decoded PQ / RaBitQ codes take it in the
// sequential order of the oracle's angular(); row traversals reduce across lanes.
template <int TRAV>
__device__ __forceinline__ float query_norm2(const float *qs, uint32_t d, int lane) {
  float qq = 0.0f;
  if (TRAV == TRAV_PQ || TRAV == TRAV_RABITQ) {
    if (lane == 0)
      for (uint32_t i = 0; i < d; ++i) qq = __fadd_rn(qq, __fmul_rn(qs[i], qs[i]));
    return __shfl_sync(kFull, qq, 0);
  }
  for (uint32_t i = lane; i < d; i += 32) qq = fmaf(qs[i], qs[i], qq);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) qq += __shfl_xor_sync(kFull, qq, o);
  return qq;
}

struct QueryCtx {
  const DgFilterOp *fops;
  uint32_t fnops;
};

// Distances for the cnt staged candidates (lane j holds cand), per traversal
// kind.  TC selects tensor-core BF16 distances (the register-list kernel);
// the general kernel, with more state per warp, computes them as packed FP32
// FMAs, which measured faster there.
template <int TRAV, int MET, int LPR, bool TC = true>
__device__ __forceinline__ float batch_distance(const SearchArgs &a, uint8_t *wsm,
                                                const WarpLayout &Ly, uint32_t cand, int cnt,
                                                int lane, float qq) {
  const float *qs = reinterpret_cast<const float *>(wsm + Ly.qf);
  const bool sqrt_l2 = a.metric == DG_L2;
  if (TRAV == TRAV_F32) {
    return rows_distance<LPR, 0, MET>(reinterpret_cast<const uint8_t *>(a.vec_f32), a.dpad * 4,
                                      (a.dpad / 4) / LPR, qs, cand, cnt, lane, sqrt_l2, qq);
  } else if (TRAV == TRAV_FP8) {
    // x = s_x e, q = s_q q': q.x = s_x s_q (e.q'); |q - x|^2 = |q|^2 + |x|^2 - 2 q.x
    const uint8_t *qhl = wsm + Ly.prov;
    const float2 qs2 = *reinterpret_cast<const float2 *>(wsm + Ly.prov + 2 * a.dpad);  // (s_q, |q|^2)
    const float2 sn = lane < cnt ? __ldg(a.fp8_sn + cand) : make_float2(0.0f, 0.0f);
    const float dot = sn.x * qs2.x * fp8_dot_mma(a.vec_fp8, a.dpad, qhl, cand, cnt, lane);
    if (MET == MET_L2) return finish_metric(MET, sqrt_l2, fmaxf(qs2.y + sn.y - 2.0f * dot, 0.0f), 0.0f, qq);
    return finish_metric(MET, false, dot, sn.y, qq);
  } else if (TRAV == TRAV_BF16 && !TC) {
    return rows_distance<LPR, 1, MET>(reinterpret_cast<const uint8_t *>(a.vec_bf16), a.dpad * 2,
                                      (a.dpad / 8) / LPR, qs, cand, cnt, lane, sqrt_l2, qq);
  } else if (TRAV == TRAV_BF16) {
    // |q - x|^2 = |q|^2 + |x|^2 - 2 q.x with q.x on the tensor cores
    const uint16_t *qhl = reinterpret_cast<const uint16_t *>(wsm + Ly.prov);
    const float q2 = *reinterpret_cast<const float *>(wsm + Ly.prov + 4 * a.dpad);
    const float xx = lane < cnt ? __ldg(a.bf16_n2 + cand) : 0.0f;
    const float dot = bf16_dot_mma(a.vec_bf16, a.dpad, qhl, cand, cnt, lane);
    if (MET == MET_L2) return finish_metric(MET, sqrt_l2, fmaxf(__fsub_rn(__fadd_rn(q2, xx), 2.0f * dot), 0.0f),
                                            0.0f, qq);
    return finish_metric(MET, false, dot, xx, qq);
  } else if (TRAV == TRAV_F16) {
    // L2 compares the f16-rounded query (F16Quantizer::prepare, src/sq.rs:51-55);
    // other metrics decode the code against the f32 query (src/quantized.rs:28-36).
    const float *qx = MET == MET_L2 ? reinterpret_cast<const float *>(wsm + Ly.prov) : qs;
    return rows_distance<LPR, 2, MET>(a.codes, a.code_stride, (a.code_stride / 16) / LPR, qx, cand,
                                      cnt, lane, sqrt_l2, qq);
  } else if (TRAV == TRAV_INT8) {
    if (MET == MET_L2) {
      const uint8_t *qc = wsm + Ly.prov;
      const uint32_t qn = *reinterpret_cast<const uint32_t *>(qc + align16(a.dpad));
      const uint32_t s = int8_l2_mma(a.codes, a.code_stride, qc, qn, a.i8_norm, cand, cnt, lane);
      float d = __fmul_rn(__fmul_rn(__uint2float_rn(s), a.i8_scale), a.i8_scale);
      return sqrt_l2 ? __fsqrt_rn(d) : d;
    } else {
      // decoded v = s c + o (src/quantized.rs:28-36, src/sq.rs decode): q.v = s (q.c) + o sum(q),
      // |v|^2 = s^2 sum(c^2) + 2 s o sum(c) + d o^2, with q.c on the tensor cores
      const uint8_t *qd = wsm + Ly.prov;
      const uint32_t ds = align16(a.dpad);
      const double2 qp = *reinterpret_cast<const double2 *>(qd + 4 * ds);  // (q scale, sum q)
      const uint32_t c2 = lane < cnt ? __ldg(a.i8_norm + cand) : 0u;
      const uint32_t c1 = lane < cnt ? __ldg(a.i8_sum + cand) : 0u;
      const double qc = int8_dot_mma(a.codes, a.code_stride, qd, ds, cand, cnt, lane) * qp.x;
      const double sc = a.i8_scale, of = a.i8_offset;
      const float dot = (float)(sc * qc + of * qp.y);
      const float vv = MET == MET_COS ? (float)(sc * sc * (double)c2 + 2.0 * sc * of * (double)c1 +
                                                (double)a.d * of * of)
                                      : 0.0f;
      return finish_metric(MET, false, dot, vv, qq);
    }
  } else if (TRAV == TRAV_PQ) {
    const float *lut = reinterpret_cast<const float *>(wsm + Ly.prov);
    float d = lane < cnt ? pq_adc(a, lut, cand) : 0.0f;
    if (MET != MET_L2)  // d = q . decode(code)
      return finish_metric(MET, false, d, (MET == MET_COS && lane < cnt) ? __ldg(a.dnorm2 + cand) : 0.0f, qq);
    return sqrt_l2 ? __fsqrt_rn(d) : d;
  } else if (MET != MET_L2) {  // RaBitQ, decoded
    const float ab = lane < cnt ? rabitq_decode_ip(a.codes + (size_t)cand * a.code_stride, a.rq_padded, wsm + Ly.prov)
                                : 0.0f;
    return finish_metric(MET, false, ab, (MET == MET_COS && lane < cnt) ? __ldg(a.dnorm2 + cand) : 0.0f, qq);
  } else {  // RaBitQ
    const uint64_t *planes = reinterpret_cast<const uint64_t *>(wsm + Ly.prov);
    const float *k5 = reinterpret_cast<const float *>(wsm + Ly.prov + 4 * (a.rq_padded / 64) * 8);
    float d = lane < cnt ? rabitq_est(a.codes + (size_t)cand * a.code_stride, a.rq_padded, planes, k5)
                         : 0.0f;
    return sqrt_l2 ? __fsqrt_rn(d) : d;
  }
}

// Stages the unvisited neighbours of an expanded node (its adjacency row) into
// stage[0..return), marking them visited.  The first 64 entries are loaded
// before any is tested, so a row of up to 64 neighbours costs one DRAM round
// trip instead of one per 32 entries.
__device__ __forceinline__ int stage_neighbours(const SearchArgs &a, const uint32_t *row, const Visited &vt,
                                                uint32_t *stage, int lane) {
  const uint32_t n0 = (uint32_t)lane < a.R ? __ldg(row + lane) : DG_PAD;
  const uint32_t n1 = (uint32_t)lane + 32 < a.R ? __ldg(row + lane + 32) : DG_PAD;
  int ns = 0;
  for (uint32_t j0 = 0; j0 < a.R; j0 += 32) {
    const uint32_t j = j0 + lane;
    const uint32_t nb = j0 == 0 ? n0 : j0 == 32 ? n1 : (j < a.R ? __ldg(row + j) : DG_PAD);
    bool ok = nb != DG_PAD && nb < a.n;
    if (ok) ok = !vt.test_and_set(nb);
    const uint32_t m = __ballot_sync(kFull, ok);
    if (ok) stage[ns + __popc(m & lanemask_lt(lane))] = nb;
    ns += __popc(m);
  }
  __syncwarp();
  return ns;
}

// Exact FP32 distance of lane j's candidate (rerank, src/quantized.rs:110-121).
template <int MET, int LPRF>
__device__ __forceinline__ float exact_distance(const SearchArgs &a, const float *qs, uint32_t cand,
                                                int cnt, int lane, float qq) {
  return rows_distance<LPRF, 0, MET>(reinterpret_cast<const uint8_t *>(a.vec_f32), a.dpad * 4,
                                     (a.dpad / 4) / LPRF, qs, cand, cnt, lane, a.metric == DG_L2, qq);
}

// Exact FP32 distance of one row by one lane (few registers): code traversals
// of a base + delta index use it for delta rows, which carry no codes
// (IncrementalDiskANN::search_with_dists scores them with distance_to,
// src/incremental.rs:955-968).  Padding columns are zero in the row and query.
template <int MET>
__device__ __forceinline__ float exact_row_distance(const SearchArgs &a, const float *qs, uint32_t id, float qq) {
  const float4 *row = reinterpret_cast<const float4 *>(a.vec_f32 + (size_t)id * a.dpad);
  const float4 *q4 = reinterpret_cast<const float4 *>(qs);
  float acc = 0.0f, bb = 0.0f;
  for (uint32_t c = 0; c < a.dpad / 4; ++c) {
    const float4 v = __ldg(row + c), q = q4[c];
    if (MET == MET_L2) {
      const float t0 = q.x - v.x, t1 = q.y - v.y, t2 = q.z - v.z, t3 = q.w - v.w;
      acc = fmaf(t0, t0, fmaf(t1, t1, fmaf(t2, t2, fmaf(t3, t3, acc))));
    } else {
      acc = fmaf(q.x, v.x, fmaf(q.y, v.y, fmaf(q.z, v.z, fmaf(q.w, v.w, acc))));
      if (MET == MET_COS) bb = fmaf(v.x, v.x, fmaf(v.y, v.y, fmaf(v.z, v.z, fmaf(v.w, v.w, bb))));
    }
  }
  return finish_metric(MET, a.metric == DG_L2, acc, bb, qq);
}

// Per-query quantizer state (QuantizerState::prepare, src/quantized.rs:167-174).
template <int TRAV, int MET>
__device__ __forceinline__ void prepare_query(const SearchArgs &a, uint8_t *wsm, const WarpLayout &Ly,
                                              const float *qs, int lane) {
  if (TRAV == TRAV_PQ && MET != MET_L2) {
    build_pq_ip_lut(a, qs, reinterpret_cast<float *>(wsm + Ly.prov), lane);
  } else if (TRAV == TRAV_RABITQ && MET != MET_L2) {
    rabitq_decode_prepare(qs, a.d, a.rq_padded, a.rq_centroid, a.rq_signs, wsm + Ly.prov, lane);
  } else if (TRAV == TRAV_PQ) {
    build_pq_lut(a, qs, reinterpret_cast<float *>(wsm + Ly.prov), lane);
  } else if (TRAV == TRAV_INT8 && MET != MET_L2) {
    // q_i ~ M t_i / F, t_i = round(q_i F / M) with F = 127 * 2^24 (M = max |q_i|),
    // split into four signed 8-bit digits t = D0 2^24 + D1 2^16 + D2 2^8 + D3
    uint8_t *dig = wsm + Ly.prov;
    const uint32_t ds = align16(a.dpad);
    float mx = 0.0f;
    double sq = 0.0;
    for (uint32_t i = lane; i < a.dpad; i += 32) {
      mx = fmaxf(mx, fabsf(qs[i]));
      sq += (double)qs[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
      sq += __shfl_xor_sync(kFull, sq, o);
    }
    const double F = 2130706432.0;  // 127 * 2^24: |t| <= F keeps D0 within [-127, 127]
    const double inv = mx > 0.0f ? F / (double)mx : 0.0;
    for (uint32_t i = lane; i < a.dpad; i += 32) {
      long long t = i < a.d ? __double2ll_rn((double)qs[i] * inv) : 0;
      int8_t dd[4];
#pragma unroll
      for (int j = 3; j > 0; --j) {
        const int dj = (int)((t + 128) & 255) - 128;
        dd[j] = (int8_t)dj;
        t = (t - dj) >> 8;
      }
      dd[0] = (int8_t)t;
#pragma unroll
      for (int j = 0; j < 4; ++j) dig[j * ds + i] = (uint8_t)dd[j];
    }
    if (lane == 0)
      *reinterpret_cast<double2 *>(dig + 4 * ds) = make_double2(mx > 0.0f ? (double)mx / F : 0.0, sq);
  } else if (TRAV == TRAV_INT8) {
    uint8_t *qc8 = wsm + Ly.prov;
    const float inv = __fdiv_rn(1.0f, a.i8_scale);
    const float beta = __fdiv_rn(-a.i8_offset, a.i8_scale);
    uint32_t qn = 0;
    for (uint32_t i = lane; i < a.dpad; i += 32) {
      const uint8_t c = i < a.d ? int8_code(qs[i], inv, beta) : 0;
      qc8[i] = c;
      qn += (uint32_t)c * c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qn += __shfl_xor_sync(kFull, qn, o);
    if (lane == 0) *reinterpret_cast<uint32_t *>(qc8 + align16(a.dpad)) = qn;
  } else if (TRAV == TRAV_FP8) {
    // scaled query q' = q / s_q (s_q = max|q| / 448) as two e4m3 columns
    uint8_t *hi = wsm + Ly.prov, *lo = hi + a.dpad;
    float mx = 0.0f, qn = 0.0f;
    for (uint32_t i = lane; i < a.dpad; i += 32) {
      mx = fmaxf(mx, fabsf(qs[i]));
      qn = fmaf(qs[i], qs[i], qn);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mx = fmaxf(mx, __shfl_xor_sync(kFull, mx, o));
      qn += __shfl_xor_sync(kFull, qn, o);
    }
    const float sq = mx > 0.0f ? __fdiv_rn(mx, 448.0f) : 1.0f;
    for (uint32_t i = lane; i < a.dpad; i += 32) {
      const float v = __fdiv_rn(qs[i], sq);
      const __nv_fp8_storage_t h = __nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
      const float hv = __half2float(__half(__nv_cvt_fp8_to_halfraw(h, __NV_E4M3)));
      hi[i] = h;
      lo[i] = __nv_cvt_float_to_fp8(__fmul_rn(__fsub_rn(v, hv), 16.0f), __NV_SATFINITE, __NV_E4M3);
    }
    if (lane == 0) *reinterpret_cast<float2 *>(wsm + Ly.prov + 2 * a.dpad) = make_float2(sq, qn);
  } else if (TRAV == TRAV_BF16) {
    // hi = bf16(q), lo = bf16(q - hi), then |q|^2 of the f32 query
    uint16_t *hi = reinterpret_cast<uint16_t *>(wsm + Ly.prov), *lo = hi + a.dpad;
    float q2 = 0.0f;
    for (uint32_t i = lane; i < a.dpad; i += 32) {
      const float v = qs[i];
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      hi[i] = __bfloat16_as_ushort(h);
      lo[i] = __bfloat16_as_ushort(__float2bfloat16_rn(__fsub_rn(v, __bfloat162float(h))));
      q2 = fmaf(v, v, q2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) q2 += __shfl_xor_sync(kFull, q2, o);
    if (lane == 0) *reinterpret_cast<float *>(wsm + Ly.prov + 4 * a.dpad) = q2;
  } else if (TRAV == TRAV_F16) {
    float *qh = reinterpret_cast<float *>(wsm + Ly.prov);
    for (uint32_t i = lane; i < a.dpad; i += 32) qh[i] = __half2float(__float2half_rn(qs[i]));
  } else if (TRAV == TRAV_RABITQ) {
    uint8_t *p = wsm + Ly.prov;
    uint64_t *planes = reinterpret_cast<uint64_t *>(p);
    float *k5 = reinterpret_cast<float *>(p + 4 * (a.rq_padded / 64) * 8);
    float *rbuf = reinterpret_cast<float *>(p + 4 * (a.rq_padded / 64) * 8 + 32);
    rabitq_prepare(qs, a.d, a.rq_padded, a.rq_centroid, a.rq_signs, rbuf, planes, k5, lane);
  }
  __syncwarp();
}

// Writes a query's results: the first k of src (sorted keys), or, with
// rerank, the first max(rerank, k) reranked with exact FP32 distances in
// their traversal order (a stable sort by exact distance, src/quantized.rs:110-121).
template <int TRAV, int MET, int LPRF>
__device__ inline void emit_results(const SearchArgs &a, uint32_t q, const uint64_t *src, int have,
                                    bool use_rerank, uint32_t search_k, uint64_t *tmp, const float *qs,
                                    float qq, uint32_t n_exp, uint32_t n_dist, int lane) {
  // this query's k; output rows are a.k apart and padded past k
  const uint32_t k = a.perK ? a.perK[q] : a.k;
  uint32_t *oid = a.out_ids + (size_t)q * a.k;
  float *od = a.out_d + (size_t)q * a.k;
  int count;
  if (use_rerank) {
    const int nr = min(have, (int)search_k);
    for (int g0 = 0; g0 < nr; g0 += 32) {
      const int cnt = min(32, nr - g0);
      const uint32_t cand = lane < cnt ? key_id(src[g0 + lane]) : 0u;
      const float d = exact_distance<MET, LPRF>(a, qs, cand, cnt, lane, qq);
      if (lane < cnt) tmp[g0 + lane] = make_key_payload(d, (uint32_t)(g0 + lane));
    }
    __syncwarp();
    warp_sort_smem(tmp, nr, lane);
    count = min(nr, (int)k);
    for (int i = lane; i < count; i += 32) {
      const uint64_t kk = tmp[i];
      oid[i] = key_id(src[key_id(kk)]);
      od[i] = key_dist(kk);
    }
  } else {
    count = min(have, (int)k);
    for (int i = lane; i < count; i += 32) {
      oid[i] = key_id(src[i]);
      od[i] = key_dist(src[i]);
    }
  }
  for (int i = count + lane; i < (int)a.k; i += 32) {
    oid[i] = DG_PAD;
    od[i] = __int_as_float(0x7f800000);
  }
  if (lane == 0) {
    a.out_cnt[q] = (uint32_t)count;
    if (a.out_stats) {
      a.out_stats[2 * q] = n_exp;
      a.out_stats[2 * q + 1] = n_dist;
    }
  }
  __syncwarp();
}

// Inserts the ns keys of skeys[] into a register-resident sorted list of at
// most 64 entries (entry i in lane i % 32: w0 for i < 32, w1 above) with
// capacity cap.  Keys not below a full list's worst entry, keys already listed
// and repeats within the batch are dropped.  Per batch of up to 32 keys the
// merge has a fixed depth: every key ranks itself within the batch (pairwise
// for a few keys, a bitonic sort for more) and within the list (binary search
// over a shared copy), its final slot is list rank + batch rank among the
// kept keys, and every output slot then gathers either its new key or the
// list entry that shifts into it.
__device__ __forceinline__ void reg_insert(const uint64_t *skeys, int ns, uint64_t &w0, uint64_t &w1, int &wsize,
                                           int cap, uint64_t *scat, uint64_t *lst, uint64_t *cst, int lane) {
  const uint32_t lt = lanemask_lt(lane);
  for (int b0 = 0; b0 < ns; b0 += 32) {
    const int cnt = min(32, ns - b0);
    uint64_t u = lane < cnt ? skeys[b0 + lane] : kKeyInvalid;
    if (wsize >= cap) {
      const uint64_t thr = strip_flag(shfl64(cap - 1 < 32 ? w0 : w1, (cap - 1) & 31));
      if (!(u < thr)) u = kKeyInvalid;
    }
    const uint32_t vm = __ballot_sync(kFull, u != kKeyInvalid);
    const int s = __popc(vm);
    if (s == 0) continue;
    // rank within the batch; repeated keys take consecutive ranks, later copies die
    int rank;
    bool dead;
    if (s > 12) {
      u = warp_sort_keys(u, lane);
      const uint64_t prev = shfl64(u, lane > 0 ? lane - 1 : 0);
      rank = lane;
      dead = lane >= s || (lane > 0 && prev == u);
    } else {
      if (u != kKeyInvalid) cst[__popc(vm & lt)] = u;
      __syncwarp();
      u = lane < s ? cst[lane] : kKeyInvalid;
      rank = 0;
      dead = lane >= s;
      for (int t = 0; t < s; ++t) {
        const uint64_t o = shfl64(u, t);
        rank += (o < u) || (o == u && t < lane);
        dead |= o == u && t < lane;
      }
    }
    // rank within the list (its stripped keys in shared memory)
    lst[lane] = strip_flag(w0);
    lst[lane + 32] = strip_flag(w1);
    __syncwarp();
    int p = 0;
#pragma unroll
    for (int step = 32; step > 0; step >>= 1)
      if (p + step <= wsize && lst[p + step - 1] < u) p += step;
    if (!dead && p < wsize && lst[p] == u) dead = true;  // already listed
    const uint32_t deadm = __reduce_or_sync(kFull, (lane < s && dead) ? (1u << rank) : 0u);
    const int na = s - __popc(deadm);
    if (na == 0) {
      __syncwarp();
      continue;
    }
    const int pos = p + rank - __popc(deadm & ((1u << (rank & 31)) - 1u));
    const bool put = !dead && pos < cap;
    const uint32_t sm0 = __reduce_or_sync(kFull, (put && pos < 32) ? (1u << pos) : 0u);
    const uint32_t sm1 = __reduce_or_sync(kFull, (put && pos >= 32) ? (1u << (pos & 31)) : 0u);
    if (put) scat[pos] = u;
    __syncwarp();
    // slot l keeps a new key, or the list entry l - (new keys before l)
    const int i0 = lane - __popc(sm0 & lt);
    const int i1 = lane + 32 - __popc(sm0) - __popc(sm1 & lt);
    const uint64_t x0 = shfl64(w0, i0 & 31), x1 = shfl64(w1, i0 & 31);
    const uint64_t y0 = shfl64(w0, i1 & 31), y1 = shfl64(w1, i1 & 31);
    const int nsz = min(cap, wsize + na);
    uint64_t n0 = ((sm0 >> lane) & 1u) ? scat[lane] : (i0 < 32 ? x0 : x1);
    uint64_t n1 = ((sm1 >> lane) & 1u) ? scat[lane + 32] : (i1 < 32 ? y0 : y1);
    w0 = lane < nsz ? n0 : kKeyInvalid;
    w1 = lane + 32 < nsz ? n1 : kKeyInvalid;
    wsize = nsz;
    __syncwarp();
  }
}

// Unfiltered search with beams up to 64: the working list lives in registers,
// entry i in lane i % 32 (w0 for i < 32, w1 above), so finding the frontier,
// the threshold and insertion ranks are ballots and shuffles instead of
// shared-memory binary searches.  Results are identical to search_one.
template <int TRAV, int MET, int LPR, int LPRF>
__device__ inline void search_one_reg(const SearchArgs &a, uint32_t q, uint8_t *wsm, const WarpLayout &Ly,
                                      int lane) {
  uint64_t *scat = reinterpret_cast<uint64_t *>(wsm + Ly.w0);  // scatter buffer, 64 keys
  uint64_t *lst = reinterpret_cast<uint64_t *>(wsm + Ly.aux);   // list copy, 64 keys
  uint64_t *skeys = reinterpret_cast<uint64_t *>(wsm + Ly.w1) ; // survivors of one expansion (<= 64)
  uint64_t *cst = reinterpret_cast<uint64_t *>(wsm + Ly.cstage);
  uint32_t *stage = reinterpret_cast<uint32_t *>(wsm + Ly.stage);
  const Visited vt{reinterpret_cast<uint32_t *>(wsm + Ly.hash), a.hbits, a.hB};
  float *qs = reinterpret_cast<float *>(wsm + Ly.qf);
  const int L = (int)(a.perL ? a.perL[q] : a.L);
  const uint32_t k = a.perK ? a.perK[q] : a.k;
  const bool use_rerank = TRAV != TRAV_F32 && a.rerank > 0;
  const uint32_t search_k = use_rerank ? max(a.rerank, k) : k;

  const float *qg = a.Q + (size_t)q * a.d;
  for (uint32_t i = lane; i < a.dpad; i += 32) qs[i] = i < a.d ? qg[i] : 0.0f;
  vt.clear(lane);
  __syncwarp();
  float qq = 0.0f;
  if (MET == MET_COS) qq = query_norm2<TRAV>(qs, a.d, lane);
  prepare_query<TRAV, MET>(a, wsm, Ly, qs, lane);

  uint64_t w0 = kKeyInvalid, w1 = kKeyInvalid;
  int wsize = 1;
  uint32_t n_exp = 0, n_dist = 1;
  {
    const uint32_t cand = a.medoid;
    float d = batch_distance<TRAV, MET, LPR>(a, wsm, Ly, cand, 1, lane, qq);
    d = __shfl_sync(kFull, d, 0);
    if (lane == 0) {
      w0 = make_key(d, cand);
      vt.test_and_set(cand);
    }
    __syncwarp();
  }
  while (true) {
    const uint32_t m0 = __ballot_sync(kFull, lane < wsize && !key_expanded(w0));
    const uint32_t m1 = __ballot_sync(kFull, lane + 32 < wsize && !key_expanded(w1));
    const int idx = m0 ? __ffs(m0) - 1 : (m1 ? 31 + __ffs(m1) : -1);
    if (idx < 0) break;
    const uint64_t best = shfl64(idx < 32 ? w0 : w1, idx & 31);
    uint64_t thr = kKeyInvalid;
    if (wsize >= L) {
      const uint64_t worst = shfl64(L - 1 < 32 ? w0 : w1, (L - 1) & 31);
      if (key_dist(best) >= key_dist(worst)) break;  // src/lib.rs:253-259
      thr = strip_flag(worst);
    }
    if (lane == (idx & 31)) {
      if (idx < 32) w0 |= 1ull;
      else w1 |= 1ull;
    }
    ++n_exp;
    // stage unvisited neighbours
    const int ns = stage_neighbours(a, a.adj + (size_t)key_id(best) * a.R, vt, stage, lane);
    n_dist += ns;
    // distances; keep only keys below the current worst (the rest cannot enter)
    int nsurv = 0;
    for (int g0 = 0; g0 < ns; g0 += 32) {
      if (nsurv > 32) {  // the 64-key survivor buffer could overflow: insert what it holds
        __syncwarp();
        reg_insert(skeys, nsurv, w0, w1, wsize, L, scat, lst, cst, lane);
        nsurv = 0;
        thr = wsize >= L ? strip_flag(shfl64(L - 1 < 32 ? w0 : w1, (L - 1) & 31)) : kKeyInvalid;
      }
      const int cnt = min(32, ns - g0);
      const uint32_t cand = lane < cnt ? stage[g0 + lane] : DG_PAD;
      const float d = batch_distance<TRAV, MET, LPR>(a, wsm, Ly, cand, cnt, lane, qq);
      const uint64_t key = lane < cnt ? make_key(d, cand) : kKeyInvalid;
      const bool sv = key < thr;
      const uint32_t m = __ballot_sync(kFull, sv);
      if (sv) skeys[nsurv + __popc(m & lanemask_lt(lane))] = key;
      nsurv += __popc(m);
    }
    __syncwarp();
    if (nsurv) reg_insert(skeys, nsurv, w0, w1, wsize, L, scat, lst, cst, lane);
  }
  // emit through the shared-memory path
  uint64_t *Wm = scat;
  if (lane < wsize) Wm[lane] = w0;
  if (lane + 32 < wsize) Wm[lane + 32] = w1;
  __syncwarp();
  emit_results<TRAV, MET, LPRF>(a, q, Wm, wsize, use_rerank, search_k, reinterpret_cast<uint64_t *>(wsm + Ly.w1),
                                qs, qq, n_exp, n_dist, lane);
}

template <int TRAV, int MET, int LPR, int LPRF, int LCAP, bool FILT>
__device__ inline void search_one(const SearchArgs &a, uint32_t q, uint8_t *wsm, const WarpLayout &Ly,
                           int lane) {
  uint64_t *W[2] = {reinterpret_cast<uint64_t *>(wsm + Ly.w0), reinterpret_cast<uint64_t *>(wsm + Ly.w1)};
  uint64_t *RES = reinterpret_cast<uint64_t *>(wsm + Ly.res);
  uint64_t *cst = reinterpret_cast<uint64_t *>(wsm + Ly.cstage);
  uint32_t *stage = reinterpret_cast<uint32_t *>(wsm + Ly.stage);
  const Visited vt{reinterpret_cast<uint32_t *>(wsm + Ly.hash), a.hbits, a.hB};
  float *qs = reinterpret_cast<float *>(wsm + Ly.qf);

  const uint32_t L = a.perL ? a.perL[q] : a.L;
  const uint32_t k = a.perK ? a.perK[q] : a.k;
  // every traversal other than exact FP32 can be reranked with FP32 rows
  const bool use_rerank = TRAV != TRAV_F32 && a.rerank > 0;
  const uint32_t search_k = use_rerank ? max(a.rerank, k) : k;

  // per-query filter program
  QueryCtx qc{a.fops, a.fnops};
  if (a.foffs) {
    qc.fops = a.fops + a.foffs[q];
    qc.fnops = a.foffs[q + 1] - a.foffs[q];
  }
  const bool labeled = FILT && qc.fnops > 0;
  const bool tombed = FILT && a.tomb != nullptr;
  const bool filtered = labeled || tombed;
  uint32_t working = L, max_iter = 0xffffffffu;
  if (labeled) {  // src/filtered.rs:35-56, src/incremental.rs:1048-1062
    working = max(L * 4, k * 10);
    max_iter = working * 2;
  } else if (tombed) {  // tombstone_config (src/incremental.rs:505-516)
    working = max(L * 2, search_k + min(a.ntomb, L));
    max_iter = working * 2;
  }
  const bool two = a.seed2 != DG_PAD && a.seed2 != a.medoid;
  if (two) working = max(working, 2u);  // both seeds enter w (src/lib.rs:218-229)

  // ---- query into shared memory (zero padded), norms, visited table
  const float *qg = a.Q + (size_t)q * a.d;
  for (uint32_t i = lane; i < a.dpad; i += 32) qs[i] = i < a.d ? qg[i] : 0.0f;
  vt.clear(lane);
  __syncwarp();
  float qq = 0.0f;
  if (MET == MET_COS) qq = query_norm2<TRAV>(qs, a.d, lane);
  prepare_query<TRAV, MET>(a, wsm, Ly, qs, lane);

  const uint64_t *labels = a.labels;
  // a result must be live (UnifiedView::is_live, src/incremental.rs:463-470) and match
  auto allow = [&](uint32_t id) -> bool {
    if (a.tomb && ((__ldg(a.tomb + (id >> 5)) >> (id & 31)) & 1u)) return false;
    return !labeled || filter_eval(qc.fops, qc.fnops, a.fpool, labels + (size_t)id * a.nf, a.nf);
  };

  // ---- seed: the medoid (DiskANN::search_with_dists seeds [medoid])
  int cur = 0, wsize = 0, rsize = 0;
  uint32_t n_exp = 0, n_dist = 0;
  // merges this lane's match key (kKeyInvalid = none) into the result list
  auto add_results = [&](uint64_t mk) {
    const int nm = prepare_batch(mk, RES, rsize, (int)search_k, cst, lane);
    if (nm > 0) {
      // merge in place through the non-current w buffer as scratch
      uint64_t *tmp = W[cur ^ 1];
      rsize = merge_keys(RES, rsize, tmp, (int)search_k, cst, nm, lane);
      for (int i = lane; i < rsize; i += 32) RES[i] = tmp[i];
      __syncwarp();
    }
  };
  // ---- seeds: the medoid, and the delta layer's entry point of a base +
  // delta index (UnifiedView::entry_points, src/incremental.rs:383-392).  They
  // are the first staged batch the loop merges (src/lib.rs:218-233).
  int ns = two ? 2 : 1;
  if (lane == 0) {
    stage[0] = a.medoid;
    vt.test_and_set(a.medoid);
    if (two) {
      stage[1] = a.seed2;
      vt.test_and_set(a.seed2);
    }
  }
  __syncwarp();

  while (true) {
    n_dist += ns;
    // ---- distances and merge, 32 candidates at a time
    for (int g0 = 0; g0 < ns; g0 += 32) {
      const int cnt = min(32, ns - g0);
      const uint32_t cand = lane < cnt ? stage[g0 + lane] : DG_PAD;
      float d = batch_distance<TRAV, MET, LPR, false>(a, wsm, Ly, cand, cnt, lane, qq);
      if (TRAV != TRAV_F32 && a.code_limit < a.n && lane < cnt && cand >= a.code_limit)
        d = exact_row_distance<MET>(a, qs, cand, qq);
      uint64_t key = lane < cnt ? make_key(d, cand) : kKeyInvalid;
      bool match = false;
      if (filtered && lane < cnt) match = allow(cand);
      insert_batch(key, W, cur, wsize, (int)working, cst, lane);
      // result list: every visited match, kept as the search_k smallest
      if (filtered) add_results((lane < cnt && match) ? make_key(d, cand) : kKeyInvalid);
    }

    // first unexpanded entry of w (the frontier minimum)
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
    const float bd = key_dist(best);
    if (filtered) {
      if (n_exp >= max_iter) break;  // src/lib.rs:237-240
      if (rsize >= (int)search_k && search_k > 0) {  // :242-251
        const float worst = key_dist(RES[search_k - 1]);
        if (worst >= 0.0f && bd > __fmul_rn(worst, 1.5f)) break;
      }
    }
    if (wsize >= (int)working && bd >= key_dist(W[cur][working - 1])) break;  // :253-259
    if (lane == 0) W[cur][idx] = best | 1ull;
    ++n_exp;

    // ---- stage unvisited neighbours
    ns = stage_neighbours(a, a.adj + (size_t)key_id(best) * a.R, vt, stage, lane);
  }

  // ---- emit
  emit_results<TRAV, MET, LPRF>(a, q, filtered ? RES : W[cur], filtered ? rsize : wsize, use_rerank, search_k,
                                W[cur ^ 1], qs, qq, n_exp, n_dist, lane);
}

// Resident blocks per SM the register allocation is sized for (4 warps each).
#ifndef DG_SEARCH_MIN_BLOCKS
#define DG_SEARCH_MIN_BLOCKS 6
#endif

template <int TRAV, int MET, int LPR, int LPRF, int LCAP, bool FILT>
__global__ void __launch_bounds__(128, DG_SEARCH_MIN_BLOCKS) beam_search_kernel(SearchArgs a, WarpLayout Ly) {
  extern __shared__ __align__(16) uint8_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *wsm = smem + (size_t)warp * Ly.total;
  while (true) {
    uint32_t q = 0;
    if (lane == 0) q = atomicAdd(a.counter, 1u);
    q = __shfl_sync(kFull, q, 0);
    if (q >= a.nq) break;
    if (a.perm) q = __ldg(a.perm + q);
    if (LCAP == 64 && !FILT)
      search_one_reg<TRAV, MET, LPR, LPRF>(a, q, wsm, Ly, lane);
    else
      search_one<TRAV, MET, LPR, LPRF, LCAP, FILT>(a, q, wsm, Ly, lane);
  }
}

}  // namespace dg
