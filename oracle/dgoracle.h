/*
 * dgoracle.h -- CPU restatement of the diskann-rs search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle for the
 * B200 kernels in pydiskann_b200.  Only the test-suite, the smoke check and
 * the CPU-baseline leg of bench.py load it; the product never links it and
 * never falls back to it.
 *
 * Every routine restates the reference algorithm at the cited lines of the
 * diskann-rs 0.5.0 sources (paths relative to the crate root).  Deliberate,
 * documented refinements:
 *   - ties between equal distances are broken by node id (lexicographic
 *     (dist, id) order) wherever the reference leaves heap order undefined;
 *   - the random draws of the graph build come from a counter-based
 *     splitmix64 stream instead of thread_rng, so a build is reproducible;
 *   - floating point is evaluated in the order written here, without FMA
 *     contraction (built with -ffp-contract=off).
 * Parity status: pinned against the known-answer tests the reference's own
 * test-suite holds (5-node beam search, filtered beam search, filter truth
 * tables, prune degree bounds, RaBitQ sizes); the reference binary itself
 * cannot be built here (no Rust toolchain), so no numeric golden vectors of
 * the reference exist.
 */
#ifndef DGORACLE_H
#define DGORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { DGO_L2SQ = 0, DGO_L2 = 1, DGO_COSINE = 2, DGO_DOT = 3 };
enum { DGO_Q_NONE = 0, DGO_Q_PQ = 1, DGO_Q_INT8 = 2, DGO_Q_RABITQ = 3, DGO_Q_F16 = 4, DGO_Q_FP8 = 5, DGO_Q_BF16 = 6 };
enum {
  DGO_F_TRUE = 0, DGO_F_EQ = 1, DGO_F_IN = 2, DGO_F_LT = 3, DGO_F_GT = 4,
  DGO_F_RANGE = 5, DGO_F_AND = 6, DGO_F_OR = 7
};
#define DGO_PAD 0xFFFFFFFFu

/* One postfix filter instruction (same encoding as DgFilterOp in dgann.h). */
typedef struct {
  uint32_t op;
  uint32_t field; /* label field for leaves, child count for AND/OR */
  uint64_t a;     /* value / min / offset into the IN value pool */
  uint64_t b;     /* max for RANGE / count for IN */
} DgoFilterOp;

typedef struct {
  uint64_t n;
  uint32_t d;
  uint32_t R;
  uint32_t medoid;
  int32_t metric;
  const float *vectors;      /* n*d */
  const uint32_t *adjacency; /* n*R, DGO_PAD padded */
  int32_t quant;
  const uint8_t *codes; /* n*code_size */
  uint32_t code_size;
  uint32_t pq_M, pq_K;
  const float *pq_codebooks; /* [M][K][d/M] */
  float int8_scale, int8_offset;
  uint32_t rq_padded;
  const float *rq_centroid; /* d */
  const float *rq_signs;    /* 3*padded */
  const uint64_t *labels;   /* n*num_fields */
  uint32_t num_fields;
  const float *fp8_scale;   /* n: per-vector scale of DGO_Q_FP8 codes (e4m3, code_size = d) */
} DgoIndex;

typedef struct {
  uint32_t k;
  uint32_t beam_width;
  uint32_t rerank_size;
  int32_t use_codes; /* traverse on quantized codes (QuantizedDiskANN) */
  const DgoFilterOp *filter;
  uint32_t filter_nops; /* 0 = Filter::None */
  const uint64_t *filter_pool;
} DgoSearchParams;

/* ---- distances (src/metric.rs:16-39) ---- */
float dgo_distance(int32_t metric, const float *a, const float *b, uint32_t d);

/* ---- counter-based random stream shared with the product build ---- */
uint64_t dgo_rand(uint64_t seed, uint64_t a, uint64_t b, uint64_t c);

/* ---- graph build (src/lib.rs:748-1073) ---- */
uint32_t dgo_medoid(const float *X, uint64_t n, uint32_t d, int32_t metric);
int dgo_robust_prune(uint32_t node, const uint32_t *cand_ids, const float *cand_d, uint32_t nc,
                     const float *X, uint32_t d, int32_t metric, uint32_t R, float alpha,
                     uint32_t *out);
int dgo_build_vamana(const float *X, uint64_t n, uint32_t d, int32_t metric, uint32_t R,
                     uint32_t Lb, float alpha, uint64_t seed, uint32_t medoid, uint32_t *adj,
                     int32_t nthreads);

/* ---- generic beam search over an explicit distance table (src/lib.rs:198-303) ---- */
int dgo_beam_search_table(const uint32_t *adj, uint32_t R, const float *node_dist,
                          const uint8_t *allow, const uint32_t *seeds, uint32_t nseeds,
                          uint32_t L, uint32_t k, int32_t filtered, uint32_t expanded,
                          uint32_t max_iter, float early_factor, uint32_t *out_ids,
                          float *out_d, uint32_t *out_n);

/* ---- index search (src/lib.rs:683-714, src/quantized.rs:68-124,300-398,
 *      src/filtered.rs:14-57) ---- */
/* IncrementalDiskANN::search_with_dists / search_filtered_with_dists
 * (src/incremental.rs:934-1070) over the unified view held in idx (base rows,
 * then delta rows): nseeds entry points, dead[id] != 0 for tombstoned rows,
 * ntomb = size of the tombstone set (selects tombstone_config, :505-516).
 * With p->use_codes (and no label filter), rows below code_limit are scored
 * by their codes and the rest exactly, then p->rerank_size reranks (:944-990). */
int dgo_incremental_search_batch(const DgoIndex *idx, const DgoSearchParams *p, const uint32_t *seeds,
                                 uint32_t nseeds, const uint8_t *dead, uint64_t ntomb, uint64_t code_limit,
                                 const float *Q, uint32_t nq, uint32_t *out_ids, float *out_d, uint32_t *out_cnt,
                                 int32_t nthreads);
int dgo_search_batch(const DgoIndex *idx, const DgoSearchParams *p, const float *Q, uint32_t nq,
                     const uint32_t *per_query_L, uint32_t *out_ids, float *out_d,
                     uint32_t *out_cnt, uint32_t *stats, int32_t nthreads);

/* ---- filter (src/filtered.rs:120-135) ---- */
int dgo_filter_matches(const DgoFilterOp *prog, uint32_t nops, const uint64_t *pool,
                       const uint64_t *labels, uint32_t num_fields);

/* ---- PQ (src/pq.rs:122-223) ---- */
void dgo_pq_encode(const float *X, uint64_t n, uint32_t d, uint32_t M, uint32_t K,
                   const float *cb, uint8_t *codes, int32_t nthreads);
void dgo_pq_lut(const float *q, uint32_t d, uint32_t M, uint32_t K, const float *cb, float *lut);
float dgo_pq_adc(const float *lut, const uint8_t *code, uint32_t M, uint32_t K);

/* ---- int8 / f16 scalar quantizers (src/sq.rs:51-229) ---- */
void dgo_int8_train(const float *X, uint64_t n, uint32_t d, float *scale, float *offset);
void dgo_int8_encode(const float *X, uint64_t n, uint32_t d, float scale, float offset,
                     uint8_t *codes);
float dgo_int8_distance(const uint8_t *q, const uint8_t *c, uint32_t d, float scale);
void dgo_f16_encode(const float *X, uint64_t n, uint32_t d, uint16_t *codes);
float dgo_f16_distance(const uint16_t *q, const uint16_t *c, uint32_t d);

/* ---- BF16 rows (the product's BF16 traversal; no counterpart in the
 *      reference): each f32 rounded to nearest even in BF16 (NaN stays NaN),
 *      code_size = 2*d; the traversal evaluates the metric of the f32 query
 *      against the decoded row, exactly as over the f32 rows ---- */
void dgo_bf16_encode(const float *X, uint64_t n, uint32_t d, uint16_t *codes);

/* ---- FP8 e4m3 with per-vector scales (the product's FP8 traversal; no
 *      counterpart in the reference): s = max|x| / 448, codes e4m3(x / s)
 *      rounded to nearest even, saturating (OCP 8-bit floating point E4M3) ---- */
uint8_t dgo_e4m3_encode(float x);
float dgo_e4m3_decode(uint8_t c);
void dgo_fp8_encode(const float *X, uint64_t n, uint32_t d, uint8_t *codes, float *scales);

/* ---- RaBitQ (src/rabitq.rs:31-256) ---- */
uint32_t dgo_rabitq_padded(uint32_t d);
void dgo_rabitq_encode(const float *X, uint64_t n, uint32_t d, uint32_t padded,
                       const float *centroid, const float *signs, uint8_t *codes);
/* q_out: [planes (4*padded/64 u64 as 8-byte words) | nq2 s k1 k2 k3 as floats] */
void dgo_rabitq_query(const float *q, uint32_t d, uint32_t padded, const float *centroid,
                      const float *signs, uint64_t *planes, float *consts5);
float dgo_rabitq_distance(const uint64_t *planes, const float *consts5, const uint8_t *code,
                          uint32_t padded);
void dgo_rabitq_distance_with_bound(const uint64_t *planes, const float *consts5,
                                    const uint8_t *code, uint32_t padded, float *est,
                                    float *err);
void dgo_rabitq_decode(const uint8_t *code, uint32_t d, uint32_t padded, const float *centroid,
                       const float *signs, float *out);

/* ---- SPFresh posting scans (src/spfresh.rs:344-378,671-770) ---- */
typedef struct {
  uint32_t d;
  int32_t metric;
  uint32_t num_blocks;
  uint32_t block_cap;
  const uint8_t *block_live;  /* num_blocks */
  const float *centroids;     /* num_blocks*d */
  const uint32_t *block_len;  /* num_blocks */
  const uint64_t *entry_ids;  /* num_blocks*block_cap */
  const uint8_t *entry_codes; /* num_blocks*block_cap*code_size */
  uint32_t code_size;
  const uint8_t *deleted; /* next_id bytes, 1 = tombstoned */
  uint64_t next_id;
  const float *raw; /* next_id*d */
  int32_t quant;
  uint32_t pq_M, pq_K;
  const float *pq_codebooks;
  float int8_scale, int8_offset;
  uint32_t rq_padded;
  const float *rq_signs;
  float probe_ratio;
  uint32_t rerank_size;
} DgoSpfresh;

int dgo_spfresh_search_batch(const DgoSpfresh *s, const float *Q, uint32_t nq, uint32_t k,
                             uint32_t nprobe, uint64_t *out_ids, float *out_d,
                             uint32_t *out_cnt, int32_t nthreads);

/* ---- exact kNN ground truth in FP64 ---- */
void dgo_exact_knn(const float *X, uint64_t n, uint32_t d, const float *Q, uint32_t nq,
                   uint32_t k, int32_t metric, uint32_t *ids, double *dists, int32_t nthreads);

#ifdef __cplusplus
}
#endif
#endif
