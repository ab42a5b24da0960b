// dg_search.cuh -- warp-per-query best-first beam search (sm_100a).
//
// Restates beam_search (diskann-rs src/lib.rs:198-303) for one query per warp:
//   * the working set `w` is a sorted shared-memory array of 64-bit keys
//     ((distance, id) order, bit 0 = "expanded");  the reference's frontier
//     min-heap is the first unexpanded entry of that array, because an entry
//     the reference evicts from `w` is never smaller than the current worst of
//     `w` and therefore only ever ends the search;
//   * one expansion gathers the adjacency row, drops visited ids, computes all
//     new distances in one batch and merges them into `w` with a warp-wide
//     bitonic sort and a merge-path scatter.  Processing a row as one batch
//     keeps exactly the L smallest (distance, id) pairs, which is what the
//     reference's sequential insert-if-smaller loop keeps;
//   * the visited set is a small exact-tag table in shared memory (struct
//     Visited).  It never reports an unvisited id as visited; an id it
//     forgets is recomputed and removed again by the duplicate check of the
//     merge (a forgotten id that is not in `w` any more cannot re-enter it,
//     since `w`'s worst entry only decreases), so results do not depend on the
//     table size;
//   * filtered search keeps the insertion-sorted result list, the iteration cap
//     and the early-termination factor of the reference's filtered branch;
//   * quantized search (src/quantized.rs:68-124) traverses on codes, then
//     reranks the first max(rerank, k) entries with exact FP32 distances in
//     their code-distance order (a stable sort by exact distance).
// Warps take queries from a global counter, so uneven beams, k and filters
// balance across the persistent grid.
#pragma once
#include "dg_common.cuh"

namespace dg {

// ------------------------------------------------------------ launch args
struct SearchArgs {
  uint64_t n;
  uint32_t d, dpad, R, medoid;
  int32_t metric;
  const float *vec_f32;   // [n][dpad] exact rows (rerank and FP32 traversal)
  const uint16_t *vec_bf16;  // [n][dpad] BF16 traversal rows (may be null)
  const float *bf16_n2;      // [n] squared norms of the BF16 rows
  const uint32_t *adj;    // [n][R]
  // quantized codes
  const uint8_t *codes;
  uint32_t code_stride;   // bytes per code row (multiple of 16)
  uint32_t pq_M, pq_K, pq_ds;
  const float *pq_cb;     // [M][K][ds]
  float i8_scale, i8_offset;
  const uint32_t *i8_norm;  // [n] sum of squared codes (int8 L2 on tensor cores)
  const uint32_t *i8_sum;   // [n] sum of codes (int8 cosine / dot on tensor cores)
  const uint8_t *vec_fp8;   // [n][dpad] e4m3 rows (FP8 traversal)
  const float2 *fp8_sn;     // [n] (scale, |decoded|^2)
  uint32_t rq_padded;
  const float *rq_centroid;  // [d]
  const float *rq_signs;     // [3][padded]
  const float *dnorm2;       // [n] squared norms of the decoded codes (cosine over PQ / RaBitQ)
  // base + delta (incremental) search: a second entry point and deleted ids
  uint32_t seed2;            // DG_PAD = one seed (the medoid)
  const uint32_t *tomb;      // [ceil(n/32)] deleted-id bitmap, null = no tombstones
  uint32_t ntomb;            // tombstone count the search config uses (> 0 when tomb is set)
  uint64_t code_limit;       // code traversals score rows >= code_limit exactly (delta rows); n = none
  // labels / filter
  const uint64_t *labels;
  uint32_t nf;
  const DgFilterOp *fops;
  const uint32_t *foffs;  // per-query program offsets (nq+1) or null
  uint32_t fnops;
  const uint64_t *fpool;
  // queries and parameters
  const float *Q;  // [nq][d]
  uint32_t nq, k, L, rerank;
  const uint32_t *perL;  // per-query L or null
  const uint32_t *perK;  // per-query k (each <= k, the output row stride) or null
  uint32_t hbits;        // log2 of the visited-table words
  uint32_t hB;           // id bits mixed by the visited table (n <= 2^hB)
  // outputs
  uint32_t *out_ids;
  float *out_d;
  uint32_t *out_cnt;
  uint32_t *out_stats;
  uint32_t *counter;  // work counter, zero at launch
  const uint32_t *perm;  // order in which the grid takes the queries (null = as given)
  uint32_t occ_pct;      // share of the resident CTAs per SM the grid uses (percent; 0 = all)
  uint32_t wpb;          // warps per CTA of the launch (1, 2 or 4; 0 = 4), one query per warp
};

enum TravKind { TRAV_F32 = 0, TRAV_BF16 = 1, TRAV_PQ = 2, TRAV_INT8 = 3, TRAV_RABITQ = 4, TRAV_F16 = 5, TRAV_FP8 = 6 };
enum MetKind { MET_L2 = 0, MET_DOT = 1, MET_COS = 2 };

constexpr int kStageCap = 256;  // max adjacency degree

// Per-warp shared-memory carve-up (byte offsets), computed on host and device.
struct WarpLayout {
  uint32_t w0, w1, res, cstage, stage, hash, qf, prov, aux, total;
};
__host__ __device__ inline uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }
// `decode`: RaBitQ or int8 with a cosine / dot metric (RaBitQ: rotated query
// and nibble table; int8: four signed digit columns of the query).
// `reg_list`: the search kernel keeps this launch's working list in registers
// (unfiltered, beams <= 64); its 32-key compaction buffer then shares the
// first 256 bytes of w0, which that path only uses as a scatter buffer
// written after every read of the compacted keys.
__host__ __device__ inline WarpLayout warp_layout(int trav, uint32_t lcap, bool filt, uint32_t hbits,
                                                  uint32_t dpad, uint32_t pq_M, uint32_t pq_K,
                                                  uint32_t rq_padded, bool decode = false,
                                                  uint32_t degree = kStageCap, bool reg_list = false) {
  WarpLayout L{};
  uint32_t o = 0;
  L.w0 = o; o += lcap * 8;
  L.w1 = o; o += lcap * 8;
  L.res = o; o += filt ? lcap * 8 : 0;
  if (reg_list && lcap == 64 && !filt) {
    L.cstage = L.w0;
  } else {
    L.cstage = o; o += 32 * 8;
  }
  L.stage = o; o += align16(max(degree, 2u) * 4);  // one adjacency row, or the two seeds
  L.hash = o; o += (1u << hbits) * 4;
  L.qf = o; o += align16(dpad * 4);
  L.prov = o;
  uint32_t p = 0;
  if (trav == TRAV_PQ) p = pq_M * pq_K * 4;
  else if (trav == TRAV_INT8 && decode) p = 4 * align16(dpad) + 16;  // query digits, then (scale, sum q)
  else if (trav == TRAV_INT8) p = align16(dpad) + 16;  // query codes, then |q_code|^2
  else if (trav == TRAV_RABITQ && decode) p = 16 + rq_padded * 4 + rq_padded * 16;
  else if (trav == TRAV_RABITQ) p = 4 * (rq_padded / 64) * 8 + 32 + align16(rq_padded * 4);
  else if (trav == TRAV_F16) p = align16(dpad * 4);
  else if (trav == TRAV_FP8) p = 2 * dpad + 16;  // query hi / lo e4m3 codes, then (scale, |q|^2)
  else if (trav == TRAV_BF16) p = 4 * dpad + 16;  // query hi / lo BF16 values, then |q|^2
  o += align16(p);
  L.aux = o;  // 64-key copy of the register-resident working list (beams <= 64)
  o += lcap == 64 && !filt ? 64 * 8 : 0;
  L.total = align16(o);
  return L;
}

// ------------------------------------------------------- small warp helpers
__device__ __forceinline__ uint32_t lanemask_lt(int lane) { return (1u << lane) - 1u; }

// ------------------------------------------------------------ visited set
// A per-query table of 2^bbits 32-bit words in shared memory, used as
// 2^(bbits-2) buckets of eight 16-bit tags (16 bytes each).  Ids are mixed by a
// multiply with an odd constant modulo 2^B (a bijection on the B-bit ids,
// n <= 2^B); the top bits of the mix pick a bucket and the remaining bits (+1,
// 0 = empty) form the tag.  A bucket keeps its eight most recent tags (a new
// tag shifts the oldest out).  (bucket, tag) identifies an id uniquely, so
// the table never reports an unvisited id as visited; it may forget an id
// when a bucket overflows, which only costs a recomputed distance.  Eight
// ways per bucket forget far fewer ids than two ways in the same bytes.  When
// the tag would need more than 15 bits the words hold whole ids instead
// (direct mapped).  Two lanes inserting into one bucket in the same
// instruction may lose one insertion (a forgotten id), never invent a tag:
// both stores carry the same shifted words and differ only in the new tag.
struct Visited {
  uint32_t *w;
  uint32_t bbits, B;
  __device__ __forceinline__ uint32_t tag_bits() const { return B - (bbits - 2); }
  __device__ __forceinline__ bool tagged() const { return tag_bits() <= 15; }
  __device__ __forceinline__ uint32_t mix(uint32_t id) const {
    const uint32_t h = id * 0x9E3779B1u;
    return B >= 32 ? h : (h & ((1u << B) - 1u));
  }
  __device__ __forceinline__ void clear(int lane) const {
    const uint32_t words = 1u << bbits, empty = tagged() ? 0u : 0xFFFFFFFFu;
    for (uint32_t i = lane; i < words; i += 32) w[i] = empty;
  }
  // True when `id` is recorded; otherwise records it.
  __device__ __forceinline__ bool test_and_set(uint32_t id) const {
    if (tagged()) {
      const uint32_t tb = tag_bits();
      const uint32_t h = mix(id);
      const uint32_t tag = (h & ((1u << tb) - 1u)) + 1u;
      uint4 *bucket = reinterpret_cast<uint4 *>(w) + (h >> tb);
      const uint4 v = *bucket;
      const uint32_t t2 = tag * 0x10001u;
      if (__vcmpeq2(v.x, t2) | __vcmpeq2(v.y, t2) | __vcmpeq2(v.z, t2) | __vcmpeq2(v.w, t2)) return true;
      *bucket = make_uint4((v.x << 16) | tag, __funnelshift_l(v.x, v.y, 16), __funnelshift_l(v.y, v.z, 16),
                           __funnelshift_l(v.z, v.w, 16));
      return false;
    }
    const uint32_t slot = (id * 0x9E3779B1u) >> (32 - bbits);
    if (w[slot] == id) return true;
    w[slot] = id;
    return false;
  }
};

// number of keys in a[0..n) that are < key (a sorted ascending)
__device__ __forceinline__ int lower_bound_smem(const uint64_t *a, int n, uint64_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Merge the nc sorted keys of cst[] into sorted src[0..size) -> dst (capacity
// cap).  Keys must be distinct nodes.  Returns the new size.
__device__ __forceinline__ int merge_keys(const uint64_t *src, int size, uint64_t *dst, int cap,
                                          const uint64_t *cst, int nc, int lane) {
  if (lane < nc) {
    uint64_t ck = cst[lane];
    int np = lower_bound_smem(src, size, ck) + lane;
    if (np < cap) dst[np] = ck;
  }
  for (int i = lane; i < size; i += 32) {
    uint64_t w = src[i];
    int np = i + lower_bound_smem(cst, nc, w);
    if (np < cap) dst[np] = w;
  }
  __syncwarp();
  return min(cap, size + nc);
}

// Given one candidate key per lane (kKeyInvalid = none), sort, drop
// duplicates within the batch and against list[0..size), drop keys that cannot
// enter a full list of capacity cap, and compact the survivors into
// cst[0..return) in ascending order.
__device__ __forceinline__ int prepare_batch(uint64_t key, const uint64_t *list, int size, int cap,
                                             uint64_t *cst, int lane) {
  key = warp_sort_keys(key, lane);
  const uint64_t prev = shfl64(key, lane > 0 ? lane - 1 : 0);
  bool ok = key != kKeyInvalid;
  if (ok && lane > 0 && prev == key) ok = false;  // duplicate id within the batch
  if (ok) {
    int pos = lower_bound_smem(list, size, key);
    if (pos < size && strip_flag(list[pos]) == key) ok = false;  // already listed
    if (size >= cap && key > strip_flag(list[cap - 1])) ok = false;  // cannot enter
  }
  const uint32_t m = __ballot_sync(kFull, ok);
  if (ok) cst[__popc(m & lanemask_lt(lane))] = key;
  __syncwarp();
  return __popc(m);
}

// Inserts one batch of candidate keys (one per lane, kKeyInvalid = none) into
// the sorted double-buffered list bufs[cur][0..size) of capacity cap.
// Keys at or above the worst entry of a full list are dropped before any
// sorting (late in a search almost every candidate is), a handful of
// survivors are ranked with shuffles, larger batches go through the warp
// bitonic sort.  Duplicates (within the batch or already listed) are dropped.
// Same result as prepare_batch + merge_keys; returns the number inserted.
__device__ __forceinline__ int insert_batch(uint64_t key, uint64_t *const bufs[2], int &cur, int &size,
                                            int cap, uint64_t *cst, int lane) {
  const uint64_t *list = bufs[cur];
  const uint64_t thr = size >= cap ? strip_flag(list[cap - 1]) : kKeyInvalid;
  const bool surv = key < thr;
  const uint32_t m = __ballot_sync(kFull, surv);
  if (!m) return 0;
  const int s = __popc(m);
  int nc;
  if (s <= 8) {
    if (surv) cst[__popc(m & lanemask_lt(lane))] = key;
    __syncwarp();
    const uint64_t k = lane < s ? cst[lane] : kKeyInvalid;
    bool alive = lane < s;
    if (alive) {
      const int pos = lower_bound_smem(list, size, k);
      if (pos < size && strip_flag(list[pos]) == k) alive = false;
    }
    for (int i = 0; i < s; ++i) {
      const uint64_t o = shfl64(k, i);
      if (i < lane && o == k) alive = false;
    }
    const uint32_t am = __ballot_sync(kFull, alive);
    int rank = 0;
    for (int i = 0; i < s; ++i) {
      const uint64_t o = shfl64(k, i);
      if (((am >> i) & 1u) && o < k) ++rank;
    }
    __syncwarp();
    if (alive) cst[rank] = k;
    __syncwarp();
    nc = __popc(am);
  } else {
    nc = prepare_batch(surv ? key : kKeyInvalid, list, size, cap, cst, lane);
  }
  if (nc > 0) {
    size = merge_keys(list, size, bufs[cur ^ 1], cap, cst, nc, lane);
    cur ^= 1;
  }
  return nc;
}

// Ascending bitonic sort of a[0..n) in shared memory by one warp (n <= 2048).
__device__ __forceinline__ void warp_sort_smem(uint64_t *a, int n, int lane) {
  int p2 = 1;
  while (p2 < n) p2 <<= 1;
  for (int i = n + lane; i < p2; i += 32) a[i] = kKeyInvalid;
  __syncwarp();
  for (int k = 2; k <= p2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < p2; i += 32) {
        int l = i ^ j;
        if (l > i) {
          uint64_t x = a[i], y = a[l];
          bool up = (i & k) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------- row-gather distances
// 16-byte read-only load of a row chunk.  With L2_256B the load asks L2 to
// fetch the whole 256-byte block around it from DRAM, so the row's later
// chunks, read by the next round of loads, hit L2 instead of paying another
// DRAM round trip: measured +13 % for FP32 rows (four rounds of 128 bytes),
// but slower for BF16 rows read by the tensor-core layout, which loads
// without it.
template <bool L2_256B>
__device__ __forceinline__ uint4 ldg_row(const uint4 *p) {
  if (L2_256B) {
    uint4 v;
    asm("ld.global.nc.L2::256B.v4.u32 {%0,%1,%2,%3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
  }
  return __ldg(p);
}

// Rows are split into 16-byte chunks; LPR lanes cooperate on one row, RPI =
// 32/LPR rows are read per warp instruction (fully coalesced), LOADS chunks
// per lane per row.  Partial sums are transposed-reduced so lane j ends up
// with candidate j's distance.
template <int ELEM>  // 0 = f32, 1 = bf16, 2 = f16
struct Chunk;
template <> struct Chunk<0> {
  static constexpr int EPC = 4;
  __device__ static void unpack(uint4 v, float (&x)[4]) {
    x[0] = __uint_as_float(v.x); x[1] = __uint_as_float(v.y);
    x[2] = __uint_as_float(v.z); x[3] = __uint_as_float(v.w);
  }
};
template <> struct Chunk<1> {
  static constexpr int EPC = 8;
  __device__ static void unpack(uint4 v, float (&x)[8]) {
    x[0] = __uint_as_float(v.x << 16); x[1] = __uint_as_float(v.x & 0xffff0000u);
    x[2] = __uint_as_float(v.y << 16); x[3] = __uint_as_float(v.y & 0xffff0000u);
    x[4] = __uint_as_float(v.z << 16); x[5] = __uint_as_float(v.z & 0xffff0000u);
    x[6] = __uint_as_float(v.w << 16); x[7] = __uint_as_float(v.w & 0xffff0000u);
  }
};
template <> struct Chunk<2> {
  static constexpr int EPC = 8;
  __device__ static void unpack(uint4 v, float (&x)[8]) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      x[2 * i] = __half2float(__ushort_as_half((unsigned short)(w[i] & 0xffffu)));
      x[2 * i + 1] = __half2float(__ushort_as_half((unsigned short)(w[i] >> 16)));
    }
  }
};

__device__ __forceinline__ float finish_metric(int met, bool sqrt_l2, float a, float b, float qq) {
  if (met == MET_L2) return sqrt_l2 ? sqrtf(a) : a;
  if (met == MET_DOT) return 1.0f - a;
  // angular (numkong): a = q.x, b = x.x, qq = q.q
  if (qq == 0.0f && b == 0.0f) return 0.0f;
  if (a == 0.0f) return 1.0f;
  float r = 1.0f - a / (sqrtf(qq) * sqrtf(b));
  return r > 0.0f ? r : 0.0f;
}

// Distance of lane j's candidate `cand` (valid when j < cnt) against the
// query held in shared memory (qs, f32, dpad long).  rows: base pointer, row
// stride in bytes; chunks = row bytes / 16.  Each round issues the loads of
// all LPR row slots before any arithmetic, so a warp keeps LPR 16-byte loads
// per lane in flight.
template <int LPR, int ELEM, int MET>
__device__ __forceinline__ float rows_distance(const uint8_t *__restrict__ rows, uint32_t stride,
                                               int loads, const float *qs, uint32_t cand, int cnt,
                                               int lane, bool sqrt_l2, float qq) {
  constexpr int RPI = 32 / LPR;
  constexpr int EPC = Chunk<ELEM>::EPC;
  const int g = lane / LPR, r = lane % LPR;
  // packed two-wide FP32 arithmetic (f32x2 FMA) within a 16-byte chunk; the
  // pair is folded into the row's running sum once per chunk
  float sa[LPR], sb[LPR];
  uint32_t ids[LPR];  // DG_PAD marks an empty slot
  const float2 neg1 = make_float2(-1.0f, -1.0f);
#pragma unroll
  for (int i = 0; i < LPR; ++i) {
    sa[i] = 0.0f;
    sb[i] = 0.0f;
    const int c = i * RPI + g;
    const uint32_t id = __shfl_sync(kFull, cand, c & 31);
    ids[i] = c < cnt ? id : DG_PAD;
  }
  for (int t = 0; t < loads; ++t) {
    const int chunk = r + LPR * t;
    uint4 v[LPR];
#pragma unroll
    for (int i = 0; i < LPR; ++i)
      if (ids[i] != DG_PAD)
        v[i] = ldg_row<ELEM == 0>(reinterpret_cast<const uint4 *>(rows + (size_t)ids[i] * stride) + chunk);
    float2 q2[EPC / 2];
#pragma unroll
    for (int e = 0; e < EPC / 2; ++e) q2[e] = reinterpret_cast<const float2 *>(qs + chunk * EPC)[e];
#pragma unroll
    for (int i = 0; i < LPR; ++i) {
      if (ids[i] != DG_PAD) {
        float x[EPC];
        Chunk<ELEM>::unpack(v[i], x);
        float2 pa = make_float2(0.0f, 0.0f), pb = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int e = 0; e < EPC / 2; ++e) {
          const float2 x2 = make_float2(x[2 * e], x[2 * e + 1]);
          if (MET == MET_L2) {
            const float2 df = __ffma2_rn(q2[e], neg1, x2);  // x - q, one rounding
            pa = __ffma2_rn(df, df, pa);
          } else {
            pa = __ffma2_rn(x2, q2[e], pa);
            if (MET == MET_COS) pb = __ffma2_rn(x2, x2, pb);
          }
        }
        sa[i] += pa.x + pa.y;
        if (MET == MET_COS) sb[i] += pb.x + pb.y;
      }
    }
  }
  float a = transpose_reduce<LPR>(sa, lane);
  float b = 0.0f;
  if (MET == MET_COS) b = transpose_reduce<LPR>(sb, lane);
  // lane l holds candidate (l % LPR) * RPI + l / LPR; route candidate j to lane j
  const int srcl = (lane % RPI) * LPR + lane / RPI;
  a = __shfl_sync(kFull, a, srcl);
  if (MET == MET_COS) b = __shfl_sync(kFull, b, srcl);
  return finish_metric(MET, sqrt_l2, a, b, qq);
}

// int8 codes: exact integer squared distance (src/sq.rs:168-172).
template <int LPR>
__device__ __forceinline__ uint32_t int8_l2_group(const uint8_t *__restrict__ codes, uint32_t stride,
                                                  int loads, const uint8_t *qcode, uint32_t cand,
                                                  int cnt, int lane) {
  constexpr int RPI = 32 / LPR;
  const int g = lane / LPR, r = lane % LPR;
  uint32_t p[LPR];
  uint32_t ids[LPR];  // DG_PAD marks an empty slot
#pragma unroll
  for (int i = 0; i < LPR; ++i) {
    p[i] = 0;
    const int c = i * RPI + g;
    const uint32_t id = __shfl_sync(kFull, cand, c & 31);
    ids[i] = c < cnt ? id : DG_PAD;
  }
  for (int t = 0; t < loads; ++t) {
    const int chunk = r + LPR * t;
    uint4 v[LPR];
#pragma unroll
    for (int i = 0; i < LPR; ++i)
      if (ids[i] != DG_PAD) v[i] = __ldg(reinterpret_cast<const uint4 *>(codes + (size_t)ids[i] * stride) + chunk);
    const uint4 qv = *reinterpret_cast<const uint4 *>(qcode + chunk * 16);
#pragma unroll
    for (int i = 0; i < LPR; ++i) {
      if (ids[i] != DG_PAD) {
        const uint32_t a0 = __vabsdiffu4(v[i].x, qv.x), a1 = __vabsdiffu4(v[i].y, qv.y);
        const uint32_t a2 = __vabsdiffu4(v[i].z, qv.z), a3 = __vabsdiffu4(v[i].w, qv.w);
        p[i] = __dp4a(a0, a0, p[i]);
        p[i] = __dp4a(a1, a1, p[i]);
        p[i] = __dp4a(a2, a2, p[i]);
        p[i] = __dp4a(a3, a3, p[i]);
      }
    }
  }
  uint32_t s = transpose_reduce<LPR>(p, lane);
  const int srcl = (lane % RPI) * LPR + lane / RPI;
  return __shfl_sync(kFull, s, srcl);
}

// One warp-wide u8 x u8 -> s32 tensor-core step (16 rows x 32 dims x 8 columns).
__device__ __forceinline__ void mma_u8_16x8x32(int (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// int8 squared distances of up to 32 candidates on the tensor cores, exact:
// |q - x|^2 = |q|^2 + |x|^2 - 2 q.x in integers.  Candidates form two tiles of
// 16 rows; lane (g = lane/4, t = lane%4) feeds rows g and g+8 of a tile.  The
// dims of every 32-wide k step are assigned per lane (any assignment works for
// a dot product as long as rows and query agree): lane t reads the 16-byte
// chunks t, t+4, t+8, ... of its rows and of the query, each chunk serving two
// k steps (bytes 0-7, then 8-15).  Every column of B holds the query, so the
// t = 0 lane of group g ends with q.x of rows g (c[0]) and g+8 (c[2]).
__device__ __forceinline__ uint32_t int8_l2_mma(const uint8_t *__restrict__ codes, uint32_t stride,
                                                const uint8_t *qcode, uint32_t qn,
                                                const uint32_t *__restrict__ xnorm, uint32_t cand, int cnt,
                                                int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int nch = (int)(stride >> 4);
  const int J = (nch + 3) >> 2;
  const uint32_t id0 = __shfl_sync(kFull, cand, 0);
  const uint32_t xn = lane < cnt ? __ldg(xnorm + cand) : 0u;  // issued first, used last
  const bool two = cnt > 16;
  // rows g, g+8 of tile 0 and (when needed) of tile 1
  const uint4 *rp[4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int row = g + 8 * h;
    uint32_t id = __shfl_sync(kFull, cand, row);
    id = row < cnt ? id : id0;
    rp[h] = reinterpret_cast<const uint4 *>(codes + (size_t)id * stride);
  }
  const uint4 *pq = reinterpret_cast<const uint4 *>(qcode);
  int c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
  const uint4 z = make_uint4(0, 0, 0, 0);
  for (int j0 = 0; j0 < J; j0 += 2) {
    uint4 x[2][4], qv[2];
    // every load of this step (both tiles) before the first tensor-core op
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int ch = t + 4 * (j0 + u);
      const bool ok = j0 + u < J && ch < nch;
#pragma unroll
      for (int h = 0; h < 4; ++h) x[u][h] = (ok && (h < 2 || two)) ? __ldg(rp[h] + ch) : z;
      qv[u] = ok ? pq[ch] : z;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      mma_u8_16x8x32(c0, x[u][0].x, x[u][1].x, x[u][0].y, x[u][1].y, qv[u].x, qv[u].y);
      mma_u8_16x8x32(c0, x[u][0].z, x[u][1].z, x[u][0].w, x[u][1].w, qv[u].z, qv[u].w);
      if (two) {
        mma_u8_16x8x32(c1, x[u][2].x, x[u][3].x, x[u][2].y, x[u][3].y, qv[u].x, qv[u].y);
        mma_u8_16x8x32(c1, x[u][2].z, x[u][3].z, x[u][2].w, x[u][3].w, qv[u].z, qv[u].w);
      }
    }
  }
  // candidate j = 16T + r sits in lane 4 * (r % 8) of tile T, row half r / 8
  const int T = lane >> 4, r = lane & 15, src = (r & 7) << 2;
  const int d00 = __shfl_sync(kFull, c0[0], src), d01 = __shfl_sync(kFull, c0[2], src);
  const int d10 = __shfl_sync(kFull, c1[0], src), d11 = __shfl_sync(kFull, c1[2], src);
  const int dot = T == 0 ? (r < 8 ? d00 : d01) : (r < 8 ? d10 : d11);
  return qn + xn - 2u * (uint32_t)dot;
}

__device__ __forceinline__ void mma_u8s8_16x8x32(int (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                                 uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k32.row.col.s32.u8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// sum_i t_i c_i for up to 32 candidate int8 code rows c, where the query enters
// as t_i = D0 2^24 + D1 2^16 + D2 2^8 + D3 with signed 8-bit digits D0..D3 held
// as four columns of the tensor-core B operand (digit j: column j; qdig: four
// arrays of dpad digits, align16(dpad) apart).  Every column product is an
// exact integer; the result is exact in double.  Tile and lane layout of
// int8_l2_mma.
__device__ __forceinline__ double int8_dot_mma(const uint8_t *__restrict__ codes, uint32_t stride,
                                               const uint8_t *qdig, uint32_t dstride, uint32_t cand, int cnt,
                                               int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int nch = (int)(stride >> 4);
  const int J = (nch + 3) >> 2;
  const uint32_t id0 = __shfl_sync(kFull, cand, 0);
  const bool two = cnt > 16;
  const uint4 *rp[4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int row = g + 8 * h;
    uint32_t id = __shfl_sync(kFull, cand, row);
    id = row < cnt ? id : id0;
    rp[h] = reinterpret_cast<const uint4 *>(codes + (size_t)id * stride);
  }
  // B column g holds digit g (columns 4..7 stay zero)
  const uint4 *pq = reinterpret_cast<const uint4 *>(qdig + (size_t)(g & 3) * dstride);
  const bool col = g < 4;
  int c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
  const uint4 z = make_uint4(0, 0, 0, 0);
  for (int j0 = 0; j0 < J; j0 += 2) {
    uint4 x[2][4], qv[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int ch = t + 4 * (j0 + u);
      const bool ok = j0 + u < J && ch < nch;
#pragma unroll
      for (int h = 0; h < 4; ++h) x[u][h] = (ok && (h < 2 || two)) ? __ldg(rp[h] + ch) : z;
      qv[u] = ok && col ? pq[ch] : z;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      mma_u8s8_16x8x32(c0, x[u][0].x, x[u][1].x, x[u][0].y, x[u][1].y, qv[u].x, qv[u].y);
      mma_u8s8_16x8x32(c0, x[u][0].z, x[u][1].z, x[u][0].w, x[u][1].w, qv[u].z, qv[u].w);
      if (two) {
        mma_u8s8_16x8x32(c1, x[u][2].x, x[u][3].x, x[u][2].y, x[u][3].y, qv[u].x, qv[u].y);
        mma_u8s8_16x8x32(c1, x[u][2].z, x[u][3].z, x[u][2].w, x[u][3].w, qv[u].z, qv[u].w);
      }
    }
  }
  // candidate j = 16T + r: row r % 8 (+8 when r >= 8) of tile T; columns 0, 1
  // sit in lane 4 (r % 8), columns 2, 3 in lane 4 (r % 8) + 1
  const int T = lane >> 4, r = lane & 15, s0 = (r & 7) << 2, hi = r >= 8 ? 2 : 0;
  int v[2][4];
#pragma unroll
  for (int tt = 0; tt < 2; ++tt) {
    const int(&c)[4] = tt == 0 ? c0 : c1;
    const int e0 = __shfl_sync(kFull, c[0], s0), e1 = __shfl_sync(kFull, c[1], s0);
    const int e2 = __shfl_sync(kFull, c[2], s0), e3 = __shfl_sync(kFull, c[3], s0);
    const int f0 = __shfl_sync(kFull, c[0], s0 + 1), f1 = __shfl_sync(kFull, c[1], s0 + 1);
    const int f2 = __shfl_sync(kFull, c[2], s0 + 1), f3 = __shfl_sync(kFull, c[3], s0 + 1);
    v[tt][0] = hi ? e2 : e0;
    v[tt][1] = hi ? e3 : e1;
    v[tt][2] = hi ? f2 : f0;
    v[tt][3] = hi ? f3 : f1;
  }
  const int *S = T == 0 ? v[0] : v[1];
  return (double)S[0] * 16777216.0 + (double)S[1] * 65536.0 + (double)S[2] * 256.0 + (double)S[3];
}

// One warp-wide BF16 x BF16 -> f32 tensor-core step (16 rows x 16 dims x 8 columns).
__device__ __forceinline__ void mma_bf16_16x8x16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                                 uint32_t a3, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// q.x for up to 32 candidate BF16 rows x on the tensor cores (FP32
// accumulate), in the tile and lane layout of int8_l2_mma: two 16-row tiles;
// lane t of group g reads the 16-byte chunks t, t+4, ... of its rows g, g+8
// (and g+16, g+24), and each chunk feeds two k steps (its first four values,
// then its last four).  The query enters as two B columns, hi = bf16(q) and
// lo = bf16(q - hi) (qhl: dpad hi values, then dpad lo values), so the result
// is x.hi + x.lo for lane j's candidate.  Every product of two BF16 values is
// exact in FP32; on integer-valued rows and queries (hi = q, lo = 0) the sums
// are exact integers below 2^24 as well.
__device__ __forceinline__ float bf16_dot_mma(const uint16_t *__restrict__ rows, uint32_t dpad,
                                              const uint16_t *qhl, uint32_t cand, int cnt, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int nch = (int)(dpad >> 3);
  const int J = (nch + 3) >> 2;
  const uint32_t id0 = __shfl_sync(kFull, cand, 0);
  const bool two = cnt > 16;
  const uint4 *rp[4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int row = g + 8 * h;
    uint32_t id = __shfl_sync(kFull, cand, row);
    id = row < cnt ? id : id0;
    rp[h] = reinterpret_cast<const uint4 *>(rows + (size_t)id * dpad);
  }
  // B column 0 holds hi, column 1 lo (columns 2..7 stay zero)
  const uint4 *pq = reinterpret_cast<const uint4 *>(qhl + (g == 1 ? dpad : 0));
  const bool col = g < 2;
  // two accumulators per tile (even and odd 16-byte chunk steps) halve the
  // chain of dependent tensor-core ops
  float c0[2][4] = {}, c1[2][4] = {};
  const uint4 z = make_uint4(0, 0, 0, 0);
  for (int j0 = 0; j0 < J; j0 += 2) {
    uint4 x[2][4], qv[2];
    // every load of this step (both tiles) before the first tensor-core op
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int ch = t + 4 * (j0 + u);
      const bool ok = j0 + u < J && ch < nch;
#pragma unroll
      for (int h = 0; h < 4; ++h)  // loads of a row's first 128 bytes fetch its whole 256-byte block into L2
        x[u][h] = (ok && (h < 2 || two)) ? (j0 == 0 ? ldg_row<true>(rp[h] + ch) : ldg_row<false>(rp[h] + ch)) : z;
      qv[u] = ok && col ? pq[ch] : z;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      mma_bf16_16x8x16(c0[u], x[u][0].x, x[u][1].x, x[u][0].y, x[u][1].y, qv[u].x, qv[u].y);
      mma_bf16_16x8x16(c0[u], x[u][0].z, x[u][1].z, x[u][0].w, x[u][1].w, qv[u].z, qv[u].w);
      if (two) {
        mma_bf16_16x8x16(c1[u], x[u][2].x, x[u][3].x, x[u][2].y, x[u][3].y, qv[u].x, qv[u].y);
        mma_bf16_16x8x16(c1[u], x[u][2].z, x[u][3].z, x[u][2].w, x[u][3].w, qv[u].z, qv[u].w);
      }
    }
  }
  // lane 4 (r % 8) of tile T holds row r % 8 (c[0], c[1]) and row r % 8 + 8
  // (c[2], c[3]) against columns hi, lo; candidate j = 16T + r
  const float a0 = __fadd_rn(__fadd_rn(c0[0][0], c0[1][0]), __fadd_rn(c0[0][1], c0[1][1]));
  const float a1 = __fadd_rn(__fadd_rn(c0[0][2], c0[1][2]), __fadd_rn(c0[0][3], c0[1][3]));
  const float b0 = __fadd_rn(__fadd_rn(c1[0][0], c1[1][0]), __fadd_rn(c1[0][1], c1[1][1]));
  const float b1 = __fadd_rn(__fadd_rn(c1[0][2], c1[1][2]), __fadd_rn(c1[0][3], c1[1][3]));
  const int T = lane >> 4, r = lane & 15, src = (r & 7) << 2;
  const float e0 = __shfl_sync(kFull, a0, src), e1 = __shfl_sync(kFull, a1, src);
  const float f0 = __shfl_sync(kFull, b0, src), f1 = __shfl_sync(kFull, b1, src);
  return T == 0 ? (r < 8 ? e0 : e1) : (r < 8 ? f0 : f1);
}

// One warp-wide e4m3 x e4m3 -> f32 tensor-core step (16 rows x 32 dims x 8 columns).
__device__ __forceinline__ void mma_e4m3_16x8x32(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                                 uint32_t a3, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k32.row.col.f32.e4m3.e4m3.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// e.q for up to 32 candidate e4m3 rows e on the tensor cores (FP32
// accumulate), in the tile and lane layout of int8_l2_mma.  The query enters
// as two e4m3 columns, hi = e4m3(q') and lo = e4m3(16 (q' - hi)) of the scaled
// query q', so the result is (e.hi + e.lo / 16) for lane j's candidate.
// qhl: hi[dpad] then lo[dpad].
__device__ __forceinline__ float fp8_dot_mma(const uint8_t *__restrict__ rows, uint32_t dpad, const uint8_t *qhl,
                                             uint32_t cand, int cnt, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int nch = (int)(dpad >> 4);
  const int J = (nch + 3) >> 2;
  const uint32_t id0 = __shfl_sync(kFull, cand, 0);
  const bool two = cnt > 16;
  const uint4 *rp[4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int row = g + 8 * h;
    uint32_t id = __shfl_sync(kFull, cand, row);
    id = row < cnt ? id : id0;
    rp[h] = reinterpret_cast<const uint4 *>(rows + (size_t)id * dpad);
  }
  // column g of B: the hi codes (g = 0), the lo codes (g = 1), zero otherwise
  const uint4 *pq = reinterpret_cast<const uint4 *>(qhl + (g == 1 ? dpad : 0));
  float c0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, c1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const uint4 z = make_uint4(0, 0, 0, 0);
  for (int j0 = 0; j0 < J; j0 += 2) {
    uint4 x[2][4], qv[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int ch = t + 4 * (j0 + u);
      const bool ok = j0 + u < J && ch < nch;
#pragma unroll
      for (int h = 0; h < 4; ++h) x[u][h] = (ok && (h < 2 || two)) ? __ldg(rp[h] + ch) : z;
      qv[u] = (ok && g < 2) ? pq[ch] : z;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      mma_e4m3_16x8x32(c0, x[u][0].x, x[u][1].x, x[u][0].y, x[u][1].y, qv[u].x, qv[u].y);
      mma_e4m3_16x8x32(c0, x[u][0].z, x[u][1].z, x[u][0].w, x[u][1].w, qv[u].z, qv[u].w);
      if (two) {
        mma_e4m3_16x8x32(c1, x[u][2].x, x[u][3].x, x[u][2].y, x[u][3].y, qv[u].x, qv[u].y);
        mma_e4m3_16x8x32(c1, x[u][2].z, x[u][3].z, x[u][2].w, x[u][3].w, qv[u].z, qv[u].w);
      }
    }
  }
  // lane 4g: c[0] / c[2] = e.hi of rows g, g+8; c[1] / c[3] = e.lo
  const int T = lane >> 4, r = lane & 15, src = (r & 7) << 2;
  const float d00 = __shfl_sync(kFull, fmaf(c0[1], 0.0625f, c0[0]), src);
  const float d01 = __shfl_sync(kFull, fmaf(c0[3], 0.0625f, c0[2]), src);
  const float d10 = __shfl_sync(kFull, fmaf(c1[1], 0.0625f, c1[0]), src);
  const float d11 = __shfl_sync(kFull, fmaf(c1[3], 0.0625f, c1[2]), src);
  return T == 0 ? (r < 8 ? d00 : d01) : (r < 8 ? d10 : d11);
}

// int8 codes decoded for non-L2 metrics (src/quantized.rs:28-36): c*scale+offset.
template <int LPR, int MET>
__device__ __forceinline__ float int8_decode_group(const uint8_t *__restrict__ codes, uint32_t stride,
                                                   int loads, const float *qs, float scale,
                                                   float offset, uint32_t dlim, uint32_t cand,
                                                   int cnt, int lane, float qq) {
  constexpr int RPI = 32 / LPR;
  const int g = lane / LPR, r = lane % LPR;
  float pa[LPR], pb[LPR];
  uint32_t ids[LPR];  // DG_PAD marks an empty slot
#pragma unroll
  for (int i = 0; i < LPR; ++i) {
    pa[i] = 0.0f;
    pb[i] = 0.0f;
    const int c = i * RPI + g;
    const uint32_t id = __shfl_sync(kFull, cand, c & 31);
    ids[i] = c < cnt ? id : DG_PAD;
  }
  for (int t = 0; t < loads; ++t) {
    const int chunk = r + LPR * t;
    uint4 v[LPR];
#pragma unroll
    for (int i = 0; i < LPR; ++i)
      if (ids[i] != DG_PAD) v[i] = __ldg(reinterpret_cast<const uint4 *>(codes + (size_t)ids[i] * stride) + chunk);
#pragma unroll
    for (int i = 0; i < LPR; ++i) {
      if (ids[i] != DG_PAD) {
        const uint32_t w[4] = {v[i].x, v[i].y, v[i].z, v[i].w};
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          // padding columns beyond the dimension decode to nothing
          float x = (uint32_t)(chunk * 16 + e) < dlim
                        ? __fadd_rn(__fmul_rn((float)((w[e >> 2] >> (8 * (e & 3))) & 0xffu), scale), offset)
                        : 0.0f;
          pa[i] = fmaf(x, qs[chunk * 16 + e], pa[i]);
          if (MET == MET_COS) pb[i] = fmaf(x, x, pb[i]);
        }
      }
    }
  }
  float a = transpose_reduce<LPR>(pa, lane);
  float b = 0.0f;
  if (MET == MET_COS) b = transpose_reduce<LPR>(pb, lane);
  const int srcl = (lane % RPI) * LPR + lane / RPI;
  a = __shfl_sync(kFull, a, srcl);
  if (MET == MET_COS) b = __shfl_sync(kFull, b, srcl);
  return finish_metric(MET, false, a, b, qq);
}

// ------------------------------------------------------------ quantizers
// PQ lookup table (src/pq.rs:181-198): lut[m][c] = sequential f32 sum of
// squared differences over the subspace, rounded like the oracle.
__device__ __forceinline__ void build_pq_lut(const SearchArgs &a, const float *qs, float *lut, int lane) {
  const uint32_t total = a.pq_M * a.pq_K;
  for (uint32_t e = lane; e < total; e += 32) {
    const uint32_t m = e / a.pq_K;
    const float *cen = a.pq_cb + (size_t)e * a.pq_ds;
    const float *qq = qs + m * a.pq_ds;
    float acc = 0.0f;
    for (uint32_t j = 0; j < a.pq_ds; ++j) {
      float t = __fsub_rn(qq[j], __ldg(cen + j));
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
    lut[e] = acc;
  }
}
// src/pq.rs:202-209: sequential f32 sum over subspaces.
__device__ __forceinline__ float pq_adc(const SearchArgs &a, const float *lut, uint32_t id) {
  const uint8_t *row = a.codes + (size_t)id * a.code_stride;
  float d = 0.0f;
  const uint32_t K = a.pq_K;
  uint32_t m = 0;
  for (uint32_t c = 0; m < a.pq_M; ++c) {
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(row) + c);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int b = 0; b < 16; ++b) {
      if (m < a.pq_M) {
        const uint32_t code = (w[b >> 2] >> (8 * (b & 3))) & 0xffu;
        d = __fadd_rn(d, lut[m * K + code]);
        ++m;
      }
    }
  }
  return d;
}

// Inner-product table for cosine / dot over PQ codes: the reference decodes
// the code (centroid concatenation, src/pq.rs:151-160) and evaluates the metric
// (src/quantized.rs:28-36); q . decode(code) = sum_m ip[m][code_m] with
// ip[m][c] = q_m . centroid(m, c).
__device__ __forceinline__ void build_pq_ip_lut(const SearchArgs &a, const float *qs, float *lut, int lane) {
  const uint32_t total = a.pq_M * a.pq_K;
  for (uint32_t e = lane; e < total; e += 32) {
    const uint32_t m = e / a.pq_K;
    const float *cen = a.pq_cb + (size_t)e * a.pq_ds;
    const float *qq = qs + m * a.pq_ds;
    float acc = 0.0f;
    for (uint32_t j = 0; j < a.pq_ds; ++j) acc = __fadd_rn(acc, __fmul_rn(qq[j], __ldg(cen + j)));
    lut[e] = acc;
  }
}

// int8 query encoding (src/sq.rs:208-220): x*(1/scale) + (-offset/scale),
// rounded to nearest even and saturated.
__device__ __forceinline__ uint8_t int8_code(float x, float inv, float beta) {
  float t = __fadd_rn(__fmul_rn(x, inv), beta);
  if (!(t == t)) return 0;
  t = rintf(t);
  if (t < 0.0f) return 0;
  if (t > 255.0f) return 255;
  return (uint8_t)t;
}

// RaBitQ query preparation (src/rabitq.rs:136-187) by one warp in shared
// memory: residual, norm, normalisation, 3 rounds of sign flip + FHT, 4-bit
// quantisation into bit planes and the estimator constants.
__device__ inline void rabitq_prepare(const float *q, uint32_t d, uint32_t P, const float *cen,
                               const float *signs, float *r, uint64_t *planes, float *k5,
                               int lane) {
  for (uint32_t i = lane; i < P; i += 32) r[i] = i < d ? __fsub_rn(q[i], cen[i]) : 0.0f;
  __syncwarp();
  float s = 0.0f;  // sequential sum of squares, as the oracle
  if (lane == 0)
    for (uint32_t i = 0; i < P; ++i) s = __fadd_rn(s, __fmul_rn(r[i], r[i]));
  const float nq = __shfl_sync(kFull, __fsqrt_rn(s), 0);
  if (nq > 0.0f)
    for (uint32_t i = lane; i < P; i += 32) r[i] = __fdiv_rn(r[i], nq);
  __syncwarp();
  for (int rd = 0; rd < 3; ++rd) {
    for (uint32_t i = lane; i < P; i += 32) r[i] = __fmul_rn(r[i], signs[rd * P + i]);
    __syncwarp();
    for (uint32_t h = 1; h < P; h *= 2) {
      for (uint32_t t = lane; t < P / 2; t += 32) {
        const uint32_t blk = t / h, off = t % h;
        const uint32_t j = blk * 2 * h + off;
        const float x = r[j], y = r[j + h];
        r[j] = __fadd_rn(x, y);
        r[j + h] = __fsub_rn(x, y);
      }
      __syncwarp();
    }
  }
  float lo = 3.402823466e38f, hi = -3.402823466e38f;
  for (uint32_t i = lane; i < P; i += 32) {
    lo = fminf(lo, r[i]);
    hi = fmaxf(hi, r[i]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(kFull, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(kFull, hi, o));
  }
  const float delta = __fdiv_rn(__fsub_rn(hi, lo), 15.0f);
  const float inv = delta > 0.0f ? __fdiv_rn(1.0f, delta) : 0.0f;
  const uint32_t words = P / 64;
  uint32_t sum_u = 0;
  for (uint32_t wd = 0; wd < words; ++wd) {
    // each lane handles 2 coordinates of this 64-bit word
    uint64_t pl[4] = {0, 0, 0, 0};
#pragma unroll
    for (int h2 = 0; h2 < 2; ++h2) {
      const uint32_t bit = lane + 32 * h2;
      const uint32_t i = wd * 64 + bit;
      float t = roundf(__fmul_rn(__fsub_rn(r[i], lo), inv));
      uint32_t u = t <= 0.0f ? 0u : (uint32_t)t;
      u = min(u, 15u);
      sum_u += u;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if ((u >> j) & 1u) pl[j] |= 1ull << bit;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      uint32_t lo32 = (uint32_t)pl[j], hi32 = (uint32_t)(pl[j] >> 32);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo32 |= __shfl_xor_sync(kFull, lo32, o);
        hi32 |= __shfl_xor_sync(kFull, hi32, o);
      }
      if (lane == 0) planes[j * words + wd] = ((uint64_t)hi32 << 32) | lo32;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum_u += __shfl_xor_sync(kFull, sum_u, o);
  if (lane == 0) {
    const float sd = __fsqrt_rn((float)P);
    k5[0] = __fmul_rn(nq, nq);
    k5[1] = __fmul_rn(2.0f, nq);
    k5[2] = __fdiv_rn(__fmul_rn(2.0f, delta), sd);
    k5[3] = __fdiv_rn(__fmul_rn(2.0f, lo), sd);
    k5[4] = __fdiv_rn(-__fadd_rn(__fmul_rn(delta, (float)sum_u), __fmul_rn((float)P, lo)), sd);
  }
  __syncwarp();
}

// src/rabitq.rs:191-197 for one code row.
__device__ __forceinline__ float rabitq_est(const uint8_t *code, uint32_t P, const uint64_t *planes,
                                            const float *k5) {
  const uint32_t words = P / 64;
  uint32_t S = 0, C = 0;
  for (uint32_t i = 0; i < words; i += 2) {
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(code) + (i >> 1));
    const uint64_t b0 = ((uint64_t)v.y << 32) | v.x;
    const uint64_t b1 = ((uint64_t)v.w << 32) | v.z;
    C += __popcll(b0);
    S += __popcll(b0 & planes[i]) + (__popcll(b0 & planes[words + i]) << 1) +
         (__popcll(b0 & planes[2 * words + i]) << 2) + (__popcll(b0 & planes[3 * words + i]) << 3);
    if (i + 1 < words) {
      C += __popcll(b1);
      S += __popcll(b1 & planes[i + 1]) + (__popcll(b1 & planes[words + i + 1]) << 1) +
           (__popcll(b1 & planes[2 * words + i + 1]) << 2) +
           (__popcll(b1 & planes[3 * words + i + 1]) << 3);
    }
  }
  const float2 nf = __ldg(reinterpret_cast<const float2 *>(code + P / 8));
  const float inner = __fadd_rn(__fadd_rn(__fmul_rn(k5[2], (float)S), __fmul_rn(k5[3], (float)C)), k5[4]);
  const float e = __fsub_rn(__fadd_rn(nf.x, k5[0]), __fmul_rn(__fmul_rn(k5[1], nf.y), inner));
  return fmaxf(e, 0.0f);
}

// ---------------------------------------------- RaBitQ decode (cosine, dot)
// The reference decodes a RaBitQ code for non-L2 metrics (src/rabitq.rs:224-238,
// src/quantized.rs:28-36): x = c + |v-c| * unrotate(b / sqrt(P)) truncated to d,
// b_i = +-1 from the sign bits.  The rotation is orthogonal (each round is a
// sign flip scaled by 1/sqrt(P) then an unnormalised Hadamard transform), so
// q . x = q . c + |v-c| * (R q) . b / sqrt(P), with R q the rotated,
// zero-padded query.  (R q) . b = 2 * sum_{b_i = 1} y_i - sum_i y_i; the masked
// sum is read from a table of the 16 subset sums of every 4 coordinates.
// Shared layout at `p`: [qc, Y, 1/sqrt(P), 0] | y[P] | T[P/4][16].
__device__ inline void rabitq_decode_prepare(const float *q, uint32_t d, uint32_t P, const float *cen,
                                             const float *signs, uint8_t *p, int lane) {
  float *hdr = reinterpret_cast<float *>(p);
  float *y = hdr + 4;
  float *T = y + P;
  float qc = 0.0f;
  for (uint32_t i = lane; i < P; i += 32) {
    const float v = i < d ? q[i] : 0.0f;
    y[i] = v;
    if (i < d) qc = fmaf(v, cen[i], qc);
  }
  __syncwarp();
  for (int rd = 0; rd < 3; ++rd) {
    for (uint32_t i = lane; i < P; i += 32) y[i] = __fmul_rn(y[i], signs[rd * P + i]);
    __syncwarp();
    for (uint32_t h = 1; h < P; h *= 2) {
      for (uint32_t t = lane; t < P / 2; t += 32) {
        const uint32_t j = (t / h) * 2 * h + t % h;
        const float x0 = y[j], x1 = y[j + h];
        y[j] = __fadd_rn(x0, x1);
        y[j + h] = __fsub_rn(x0, x1);
      }
      __syncwarp();
    }
  }
  float Y = 0.0f;
  for (uint32_t i = lane; i < P; i += 32) Y += y[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Y += __shfl_xor_sync(kFull, Y, o);
    qc += __shfl_xor_sync(kFull, qc, o);
  }
  for (uint32_t e = lane; e < P * 4; e += 32) {
    const uint32_t j = e >> 4, nib = e & 15u;
    float t = 0.0f;
#pragma unroll
    for (int b = 0; b < 4; ++b)
      if ((nib >> b) & 1u) t = __fadd_rn(t, y[4 * j + b]);
    T[e] = t;
  }
  if (lane == 0) {
    hdr[0] = qc;
    hdr[1] = Y;
    hdr[2] = __fdiv_rn(1.0f, __fsqrt_rn((float)P));
    hdr[3] = 0.0f;
  }
  __syncwarp();
}

// q . decode(code) for one code (one lane).
__device__ __forceinline__ float rabitq_decode_ip(const uint8_t *code, uint32_t P, const uint8_t *p) {
  const float *hdr = reinterpret_cast<const float *>(p);
  const float *T = hdr + 4 + P;
  float s1 = 0.0f;
  for (uint32_t c = 0; c < P / 128; ++c) {
    const uint4 v = __ldg(reinterpret_cast<const uint4 *>(code) + c);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int nb = 0; nb < 8; ++nb) s1 += T[((c * 4 + k) * 8 + nb) * 16 + ((w[k] >> (4 * nb)) & 15u)];
  }
  if (P % 128) {  // P = 64: one 8-byte word
    const uint2 v = __ldg(reinterpret_cast<const uint2 *>(code + (P / 128) * 16));
    const uint32_t w[2] = {v.x, v.y};
    const uint32_t base = (P / 128) * 32;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
      for (int nb = 0; nb < 8; ++nb) s1 += T[(base + k * 8 + nb) * 16 + ((w[k] >> (4 * nb)) & 15u)];
  }
  const float n2 = __ldg(reinterpret_cast<const float *>(code + P / 8));
  const float ip = (2.0f * s1 - hdr[1]) * hdr[2];
  return hdr[0] + sqrtf(n2) * ip;
}

}  // namespace dg
