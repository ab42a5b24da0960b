// dg_search_kernel.cuh -- the persistent beam-search kernel template.
#pragma once
#include "dg_search.cuh"

namespace dg {

struct QueryCtx {
  const DgFilterOp *fops;
  uint32_t fnops;
};

// Distances for the cnt staged candidates (lane j holds cand), per traversal kind.
template <int TRAV, int MET, int LPR>
__device__ __forceinline__ float batch_distance(const SearchArgs &a, uint8_t *wsm,
                                                const WarpLayout &Ly, uint32_t cand, int cnt,
                                                int lane, float qq) {
  const float *qs = reinterpret_cast<const float *>(wsm + Ly.qf);
  const bool sqrt_l2 = a.metric == DG_L2;
  if (TRAV == TRAV_F32) {
    return rows_distance<LPR, 0, MET>(reinterpret_cast<const uint8_t *>(a.vec_f32), a.dpad * 4,
                                      (a.dpad / 4) / LPR, qs, cand, cnt, lane, sqrt_l2, qq);
  } else if (TRAV == TRAV_BF16) {
    return rows_distance<LPR, 1, MET>(reinterpret_cast<const uint8_t *>(a.vec_bf16), a.dpad * 2,
                                      (a.dpad / 8) / LPR, qs, cand, cnt, lane, sqrt_l2, qq);
  } else if (TRAV == TRAV_F16) {
    // L2 compares the f16-rounded query (F16Quantizer::prepare, src/sq.rs:51-55);
    // other metrics decode the code against the f32 query (src/quantized.rs:28-36).
    const float *qx = MET == MET_L2 ? reinterpret_cast<const float *>(wsm + Ly.prov) : qs;
    return rows_distance<LPR, 2, MET>(a.codes, a.code_stride, (a.code_stride / 16) / LPR, qx, cand,
                                      cnt, lane, sqrt_l2, qq);
  } else if (TRAV == TRAV_INT8) {
    if (MET == MET_L2) {
      const uint8_t *qc = wsm + Ly.prov;
      uint32_t s = int8_l2_group<LPR>(a.codes, a.code_stride, (a.code_stride / 16) / LPR, qc, cand,
                                      cnt, lane);
      float d = __fmul_rn(__fmul_rn(__uint2float_rn(s), a.i8_scale), a.i8_scale);
      return sqrt_l2 ? __fsqrt_rn(d) : d;
    } else {
      return int8_decode_group<LPR, MET>(a.codes, a.code_stride, (a.code_stride / 16) / LPR, qs,
                                         a.i8_scale, a.i8_offset, a.d, cand, cnt, lane, qq);
    }
  } else if (TRAV == TRAV_PQ) {
    const float *lut = reinterpret_cast<const float *>(wsm + Ly.prov);
    float d = lane < cnt ? pq_adc(a, lut, cand) : 0.0f;
    return sqrt_l2 ? __fsqrt_rn(d) : d;
  } else {  // RaBitQ
    const uint64_t *planes = reinterpret_cast<const uint64_t *>(wsm + Ly.prov);
    const float *k5 = reinterpret_cast<const float *>(wsm + Ly.prov + 4 * (a.rq_padded / 64) * 8);
    float d = lane < cnt ? rabitq_est(a.codes + (size_t)cand * a.code_stride, a.rq_padded, planes, k5)
                         : 0.0f;
    return sqrt_l2 ? __fsqrt_rn(d) : d;
  }
}

// Exact FP32 distance of lane j's candidate (rerank, src/quantized.rs:110-121).
template <int MET, int LPRF>
__device__ __forceinline__ float exact_distance(const SearchArgs &a, const float *qs, uint32_t cand,
                                                int cnt, int lane, float qq) {
  return rows_distance<LPRF, 0, MET>(reinterpret_cast<const uint8_t *>(a.vec_f32), a.dpad * 4,
                                     (a.dpad / 4) / LPRF, qs, cand, cnt, lane, a.metric == DG_L2, qq);
}

__device__ __forceinline__ uint32_t vhash(uint32_t id, uint32_t hbits) {
  return (id * 2654435761u) >> (32 - hbits);
}

template <int TRAV, int MET, int LPR, int LPRF, int LCAP, bool FILT>
__device__ inline void search_one(const SearchArgs &a, uint32_t q, uint8_t *wsm, const WarpLayout &Ly,
                           int lane) {
  uint64_t *W[2] = {reinterpret_cast<uint64_t *>(wsm + Ly.w0), reinterpret_cast<uint64_t *>(wsm + Ly.w1)};
  uint64_t *RES = reinterpret_cast<uint64_t *>(wsm + Ly.res);
  uint64_t *cst = reinterpret_cast<uint64_t *>(wsm + Ly.cstage);
  uint32_t *stage = reinterpret_cast<uint32_t *>(wsm + Ly.stage);
  uint32_t *hash = reinterpret_cast<uint32_t *>(wsm + Ly.hash);
  float *qs = reinterpret_cast<float *>(wsm + Ly.qf);
  const uint32_t hsz = 1u << a.hbits;

  const uint32_t L = a.perL ? a.perL[q] : a.L;
  const uint32_t k = a.k;
  // every traversal other than exact FP32 can be reranked with FP32 rows
  const bool use_rerank = TRAV != TRAV_F32 && a.rerank > 0;
  const uint32_t search_k = use_rerank ? max(a.rerank, k) : k;

  // per-query filter program
  QueryCtx qc{a.fops, a.fnops};
  if (a.foffs) {
    qc.fops = a.fops + a.foffs[q];
    qc.fnops = a.foffs[q + 1] - a.foffs[q];
  }
  const bool filtered = FILT && qc.fnops > 0;
  uint32_t working = L, max_iter = 0xffffffffu;
  if (filtered) {  // src/filtered.rs:35-56
    working = max(L * 4, k * 10);
    max_iter = working * 2;
  }

  // ---- query into shared memory (zero padded), norms, visited table
  const float *qg = a.Q + (size_t)q * a.d;
  for (uint32_t i = lane; i < a.dpad; i += 32) qs[i] = i < a.d ? qg[i] : 0.0f;
  for (uint32_t i = lane; i < hsz; i += 32) hash[i] = DG_PAD;
  __syncwarp();
  float qq = 0.0f;
  if (MET == MET_COS) {
    for (uint32_t i = lane; i < a.dpad; i += 32) qq = fmaf(qs[i], qs[i], qq);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) qq += __shfl_xor_sync(kFull, qq, o);
  }
  // ---- per-query quantizer state (QuantizerState::prepare, src/quantized.rs:167-174)
  if (TRAV == TRAV_PQ) {
    build_pq_lut(a, qs, reinterpret_cast<float *>(wsm + Ly.prov), lane);
  } else if (TRAV == TRAV_INT8) {
    uint8_t *qc8 = wsm + Ly.prov;
    const float inv = __fdiv_rn(1.0f, a.i8_scale);
    const float beta = __fdiv_rn(-a.i8_offset, a.i8_scale);
    for (uint32_t i = lane; i < a.dpad; i += 32) qc8[i] = i < a.d ? int8_code(qs[i], inv, beta) : 0;
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

  const uint64_t *labels = a.labels;
  auto allow = [&](uint32_t id) -> bool {
    return filter_eval(qc.fops, qc.fnops, a.fpool, labels + (size_t)id * a.nf, a.nf);
  };

  // ---- seed: the medoid (DiskANN::search_with_dists seeds [medoid])
  int cur = 0, wsize = 0, rsize = 0;
  uint32_t n_exp = 0, n_dist = 0;
  {
    const uint32_t cand = a.medoid;
    float d = batch_distance<TRAV, MET, LPR>(a, wsm, Ly, cand, 1, lane, qq);
    d = __shfl_sync(kFull, d, 0);
    if (lane == 0) {
      W[0][0] = make_key(d, cand);
      hash[vhash(cand, a.hbits)] = cand;
      if (filtered && allow(cand)) RES[0] = make_key(d, cand);
    }
    wsize = 1;
    if (filtered) rsize = __shfl_sync(kFull, (lane == 0 && allow(cand)) ? 1 : 0, 0);
    n_dist = 1;
    __syncwarp();
  }

  while (true) {
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
    const uint32_t node = key_id(best);
    const uint32_t *row = a.adj + (size_t)node * a.R;
    int ns = 0;
    for (uint32_t j0 = 0; j0 < a.R; j0 += 32) {
      const uint32_t j = j0 + lane;
      uint32_t nb = j < a.R ? __ldg(row + j) : DG_PAD;
      bool ok = nb != DG_PAD && nb < a.n;
      if (ok) ok = hash[vhash(nb, a.hbits)] != nb;
      const uint32_t m = __ballot_sync(kFull, ok);
      if (ok) {
        stage[ns + __popc(m & lanemask_lt(lane))] = nb;
        hash[vhash(nb, a.hbits)] = nb;
      }
      ns += __popc(m);
    }
    __syncwarp();
    n_dist += ns;

    // ---- distances and merge, 32 candidates at a time
    for (int g0 = 0; g0 < ns; g0 += 32) {
      const int cnt = min(32, ns - g0);
      const uint32_t cand = lane < cnt ? stage[g0 + lane] : DG_PAD;
      const float d = batch_distance<TRAV, MET, LPR>(a, wsm, Ly, cand, cnt, lane, qq);
      uint64_t key = lane < cnt ? make_key(d, cand) : kKeyInvalid;
      bool match = false;
      if (filtered && lane < cnt) match = allow(cand);
      insert_batch(key, W, cur, wsize, (int)working, cst, lane);
      if (filtered) {
        // result list: every visited match, kept as the search_k smallest
        uint64_t mk = (lane < cnt && match) ? make_key(d, cand) : kKeyInvalid;
        const int nm = prepare_batch(mk, RES, rsize, (int)search_k, cst, lane);
        if (nm > 0) {
          // merge in place through the non-current w buffer as scratch
          uint64_t *tmp = W[cur ^ 1];
          rsize = merge_keys(RES, rsize, tmp, (int)search_k, cst, nm, lane);
          for (int i = lane; i < rsize; i += 32) RES[i] = tmp[i];
          __syncwarp();
        }
      }
    }
  }

  // ---- emit
  const uint64_t *src = filtered ? RES : W[cur];
  const int have = filtered ? rsize : wsize;
  uint32_t *oid = a.out_ids + (size_t)q * k;
  float *od = a.out_d + (size_t)q * k;
  int count;
  if (use_rerank) {
    const int nr = min(have, (int)search_k);
    uint64_t *tmp = W[cur ^ 1];
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
  for (int i = count + lane; i < (int)k; i += 32) {
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
    search_one<TRAV, MET, LPR, LPRF, LCAP, FILT>(a, q, wsm, Ly, lane);
  }
}

}  // namespace dg
