/*
 * dgann.h -- C ABI of libdgann, the B200 (sm_100a) search hot path of
 * pydiskann_b200: batched Vamana/DiskANN beam search (FP32 / BF16 storage,
 * PQ, int8 SQ, F16 and RaBitQ codes with an exact FP32 rerank), label-filtered
 * beam search and SPFresh posting-list scans.
 *
 * The entry points replace the search surface of diskann-rs 0.5.0 (paths
 * relative to the crate root; each declaration names what it stands in for).
 * Conventions:
 *   - every call returns a DgStatus; DG_OK is 0.  On failure the thread-local
 *     message of dg_last_error() says why.  Nothing panics or throws across
 *     the ABI (the reference asserts on a dimension mismatch,
 *     src/lib.rs:684-690; here that is DG_EINVAL).
 *   - ids are u32 node ids (u64 for SPFresh); result rows are k-strided and
 *     padded with DG_PAD / +inf; the true count of each row is in out_counts
 *     (the reference returns min(k, found), tests/correctness.rs:58-66).
 *   - the caller owns every input; dg_*_create copies what it needs into HBM.
 *     Query and output pointers are host memory unless DG_FLAG_DEVICE_PTRS is
 *     set, in which case they are device pointers on the handle's device.
 *   - a handle may be searched from several host threads; calls on one handle
 *     are serialised internally.  `stream` (a cudaStream_t, may be NULL for the
 *     handle's own stream) orders the work; with host pointers the call
 *     returns after the results are in host memory.
 */
#ifndef DGANN_H
#define DGANN_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DG_API __attribute__((visibility("default")))
#else
#define DG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DG_PAD 0xFFFFFFFFu
#define DG_PAD64 0xFFFFFFFFFFFFFFFFull
#define DGANN_VERSION 1

typedef enum {
  DG_OK = 0,
  DG_EINVAL = 1,   /* bad shape, dimension mismatch, bad parameter */
  DG_ENOMEM = 2,   /* HBM budget exceeded / allocation failed */
  DG_ETIMEOUT = 3, /* a bounded device wait expired */
  DG_EDEVICE = 4,  /* CUDA error (message in dg_last_error) */
  DG_ENOTSUP = 5   /* combination not implemented */
} DgStatus;

/* Metrics (src/metric.rs:16-39; the Python binding's "l2" is squared L2,
 * python/src/lib.rs:13,28). */
typedef enum { DG_L2SQ = 0, DG_L2 = 1, DG_COSINE = 2, DG_DOT = 3 } DgMetric;

/* Where the beam search takes its distances from. */
typedef enum {
  DG_TRAVERSE_F32 = 0,  /* full vectors (DiskANN::distance_to, src/lib.rs:726-733) */
  DG_TRAVERSE_BF16 = 1, /* BF16 copy of the vectors, FP32 accumulate */
  DG_TRAVERSE_CODES = 2, /* quantized codes (QuantizedDiskANN, src/quantized.rs:13-54) */
  DG_TRAVERSE_FP8 = 3    /* FP8 e4m3 copy with per-vector scales, FP32 accumulate (dg_index_enable_fp8) */
} DgTraversal;

typedef enum { DG_Q_NONE = 0, DG_Q_PQ = 1, DG_Q_INT8 = 2, DG_Q_RABITQ = 3, DG_Q_F16 = 4 } DgQuantizer;

/* Filter::matches as a postfix program (src/filtered.rs:61-135). Leaves test
 * labels[field] (a missing field never matches); AND/OR pop `field` results. */
typedef enum {
  DG_F_TRUE = 0, DG_F_EQ = 1, DG_F_IN = 2, DG_F_LT = 3, DG_F_GT = 4,
  DG_F_RANGE = 5, DG_F_AND = 6, DG_F_OR = 7
} DgFilterOpCode;
typedef struct {
  uint32_t op;
  uint32_t field; /* label field of a leaf; child count of AND/OR */
  uint64_t a;     /* value (EQ/LT/GT), min (RANGE), offset into the value pool (IN) */
  uint64_t b;     /* max (RANGE), value count (IN) */
} DgFilterOp;

#define DG_FLAG_DEVICE_PTRS 1u /* queries / outputs are device pointers */
#define DG_FLAG_STREAM 2u      /* run on `stream` as given; NULL = the legacy default stream */

typedef struct DgIndex DgIndex;

/* Graph index: replaces DiskANN<D> (src/lib.rs:305-330) once built/opened. */
typedef struct {
  uint32_t dim;
  uint32_t max_degree; /* R; adjacency rows are R slots padded with DG_PAD */
  uint64_t num_vectors;
  uint32_t medoid;     /* entry point (src/lib.rs:748-768) */
  int32_t metric;      /* DgMetric */
  const float *vectors;      /* host f32[num_vectors*dim] */
  const uint32_t *adjacency; /* host u32[num_vectors*max_degree] */
  int32_t device;            /* CUDA device ordinal */
  uint64_t hbm_budget_bytes; /* 0 = no limit; creation fails with DG_ENOMEM beyond it */
} DgIndexDesc;

/* DiskANN::build_index / open -> a device-resident index. */
DG_API DgStatus dg_index_create(const DgIndexDesc *desc, DgIndex **out);
DG_API DgStatus dg_index_destroy(DgIndex *idx);

/* Adds a BF16 copy of the vectors for DG_TRAVERSE_BF16 (FP32 accumulate). */
DG_API DgStatus dg_index_enable_bf16(DgIndex *idx);

/* Adds an FP8 (e4m3) copy of the vectors for DG_TRAVERSE_FP8: per vector a
 * scale s = max|x| / 448 and codes e4m3(x / s) (round to nearest even,
 * saturating), plus |s * e4m3(x / s)|^2.  No counterpart in the reference: a
 * lower-precision traversal that, like BF16, is meant to be followed by the
 * exact FP32 rerank (rerank_size). */
DG_API DgStatus dg_index_enable_fp8(DgIndex *idx);

/* QuantizedDiskANN::from_pq (src/quantized.rs:210-222): codebooks
 * [M][K][dim/M] f32, codes u8[n*M].  Pass codes = NULL to encode on the GPU
 * with ProductQuantizer::encode semantics (src/pq.rs:122-149). */
DG_API DgStatus dg_index_attach_pq(DgIndex *idx, uint32_t M, uint32_t K, const float *codebooks,
                            const uint8_t *codes);
/* QuantizedDiskANN::from_int8 (src/quantized.rs:252-265): global scale/offset
 * (src/sq.rs:128-157); codes = NULL encodes on the GPU (src/sq.rs:208-220). */
DG_API DgStatus dg_index_attach_int8(DgIndex *idx, float scale, float offset, const uint8_t *codes);
/* QuantizedDiskANN::from_f16 (src/quantized.rs:225-236). */
DG_API DgStatus dg_index_attach_f16(DgIndex *idx);
/* The same with the codes given: u16[n*dim] f16 bit patterns, as a QANN
 * sidecar stores them (src/quantized.rs:490-509); NULL encodes on the GPU. */
DG_API DgStatus dg_index_attach_f16_codes(DgIndex *idx, const uint8_t *codes);
/* QuantizedDiskANN::from_rabitq (src/quantized.rs:239-249): padded dim,
 * centroid f32[dim], signs f32[3*padded] (src/rabitq.rs:78-107); codes of
 * padded/8+8 bytes or NULL to encode on the GPU (src/rabitq.rs:218-256). */
DG_API DgStatus dg_index_attach_rabitq(DgIndex *idx, uint32_t padded, const float *centroid,
                                const float *signs, const uint8_t *codes);
/* FilteredDiskANN labels (src/filtered.rs:140-160): u64[n*num_fields]. */
DG_API DgStatus dg_index_attach_labels(DgIndex *idx, uint32_t num_fields, const uint64_t *labels);
/* Base + delta (incremental) search, IncrementalDiskANN (src/incremental.rs):
 * the index holds the unified view's rows -- base rows, then delta rows, then
 * spare capacity (unreachable until rows are written) -- with adjacency rows of
 * max_degree slots (UnifiedView, :349-471).
 *
 * Entry points: ids[0] (the base medoid) and optionally ids[1] (base count +
 * the delta layer's entry point), seeded as UnifiedView::entry_points
 * (:383-392). */
DG_API DgStatus dg_index_set_entry_points(DgIndex *idx, const uint32_t *ids, uint32_t n);
/* Marks (deleted = 1) or clears unified ids in the tombstone bitmap; results
 * skip marked ids (is_live, :463-470) and, while tombstone_count > 0, searches
 * use tombstone_config (:505-516): expanded beam max(2L, k + min(count, L)),
 * 2x iterations, early-termination factor 1.5.  tombstone_count is the size
 * of the caller's tombstone set (which may hold ids the index does not have).
 * This call and dg_index_update_rows rewrite device state only after every
 * dg_search_batch already issued (on any stream) has finished, as the
 * reference's searches hold a read lock for their whole run; the GPU orders
 * them and the host does not wait.  dg_search_batch_static calls are the
 * caller's to order. */
DG_API DgStatus dg_index_set_tombstones(DgIndex *idx, const uint32_t *ids, uint64_t n, int32_t deleted,
                                        uint64_t tombstone_count);
/* Rows at or past `limit` carry no codes: code traversals score them with the
 * exact FP32 distance, as IncrementalDiskANN::search_with_dists scores delta
 * rows of a quantized base (src/incremental.rs:944-968).  limit = 0 or n:
 * every row is coded (the default). */
DG_API DgStatus dg_index_set_code_limit(DgIndex *idx, uint64_t limit);
/* Overwrites rows [first, first + count): f32 vectors (dim each; BF16 / FP8
 * copies are re-encoded), adjacency (max_degree each) and labels (num_fields
 * each); a NULL pointer leaves that part unchanged.  Vectors of rows that
 * carry quantized codes cannot be replaced (DG_ENOTSUP); rows past the code
 * limit can. */
DG_API DgStatus dg_index_update_rows(DgIndex *idx, uint64_t first, uint64_t count, const float *vectors,
                                     const uint32_t *adjacency, const uint64_t *labels);
/* DeltaLayer::add_vectors (src/incremental.rs:114-166) on the host: inserts
 * rows [n_old, n_old + n_new) of `vectors` ([n][dim] f32) into the delta graph
 * `adjacency` ([n][max_degree] u32, DG_PAD padded, lists in the reference's
 * order), each by greedy search from the entry point (beam max(2R, 16)),
 * alpha-pruning (robust_prune, alpha 1.2, src/lib.rs:977-1034) and back-edges
 * (pruned when a list is full); *entry_point (-1 = none) becomes the medoid
 * of all rows (compute_medoid, :168-193) when more than one row exists. */
DG_API DgStatus dg_delta_insert(const float *vectors, uint32_t dim, int32_t metric, uint32_t max_degree,
                                uint32_t *adjacency, uint64_t n_old, uint64_t n_new, int64_t *entry_point);

/* The attached quantizer's codes, n rows of code_size bytes in the layout the
 * QANN sidecar stores (QuantizedDiskANN::quantized_to_bytes, src/quantized.rs:
 * 490-509); out = NULL only reports code_size.  Lets a caller persist an index
 * whose codes were encoded on the GPU. */
DG_API DgStatus dg_index_get_codes(DgIndex *idx, uint8_t *out, uint64_t out_len, uint32_t *code_size);

typedef struct {
  uint32_t k;
  uint32_t beam_width;  /* L (search_with_dists' beam_width) */
  uint32_t rerank_size; /* QuantizedConfig::rerank_size (src/quantized.rs:133-143) */
  int32_t traversal;    /* DgTraversal */
  /* Filter: ops[filter_offsets[q] .. filter_offsets[q+1]) is query q's
   * program when filter_offsets != NULL; otherwise ops[0..filter_nops) applies
   * to every query; no ops = Filter::None. Host pointers. */
  const DgFilterOp *filter_ops;
  uint32_t filter_nops;
  const uint32_t *filter_offsets;
  const uint64_t *filter_pool;
  uint32_t filter_pool_len;
  const uint32_t *per_query_beam; /* optional u32[nq] host array of per-query L */
  uint32_t flags;                 /* DG_FLAG_* */
  void *stream;                   /* cudaStream_t; without DG_FLAG_STREAM, NULL = the handle's stream */
  /* optional u32[nq] host array of per-query k, each in [1, k]: query q
   * returns up to per_query_k[q] results in its output row, which stays k
   * entries long (padded with 0xFFFFFFFF / +inf past its count) */
  const uint32_t *per_query_k;
} DgSearchParams;

/* Batched search.  Stands in for DiskANN::search_with_dists (src/lib.rs:683-714),
 * QuantizedDiskANN::search_with_dists / search_batch /
 * search_filtered_with_dists (src/quantized.rs:300-398) and
 * FilteredDiskANN::search_filtered_with_dists / search_filtered_batch
 * (src/filtered.rs:436-480).  queries f32[nq*dim]; out_ids u32[nq*k];
 * out_dists f32[nq*k]; out_counts u32[nq]; out_stats (optional) u32[nq*2] =
 * (expansions, distance evaluations) per query. */
DG_API DgStatus dg_search_batch(DgIndex *idx, const DgSearchParams *p, const float *queries, uint32_t nq,
                         uint32_t *out_ids, float *out_dists, uint32_t *out_counts,
                         uint32_t *out_stats);

/* Launch-schedule autotuner (no counterpart in the reference): times this
 * exact search -- the caller's parameters and queries (host or device per
 * p->flags) -- under candidate launch schedules and keeps the fastest for
 * later searches of the same traversal, working-set capacity and filtering.
 * The axes, searched one after another: the per-query visited-table size
 * from 2^8 to 2^13 words (its shared memory sets how many queries an SM
 * holds; a smaller table recomputes the distances of ids it forgets), the
 * order in which the persistent grid takes the queries (as given, or grouped
 * by nearest pivot row so that queries in one region of the graph run
 * together and share rows in L2), the share of the resident CTAs per SM
 * the grid uses (100, 75, 50 %), and the warps (queries in flight) per CTA
 * (4, 2, 1: a query with a large state -- long beams, wide rows -- packs an
 * SM's shared memory more finely in smaller CTAs).  No schedule changes a
 * result.
 * ms_per_call[6] (may be NULL) receives the mean time per call of each table
 * size, -1 where the size did not fit in shared memory. */
DG_API DgStatus dg_index_autotune(DgIndex *idx, const DgSearchParams *p, const float *queries, uint32_t nq,
                                  uint32_t reps, uint32_t *best_hbits, float *ms_per_call);
/* The schedule the last dg_index_autotune chose: visited-table bits, query
 * order (0 = as given, 1 = grouped by nearest pivot), percent of the
 * resident CTAs per SM and warps per CTA (each out pointer may be NULL).  No
 * counterpart in the reference. */
DG_API DgStatus dg_index_tuned_schedule(DgIndex *idx, uint32_t *hbits, uint32_t *order, uint32_t *occ_pct,
                                        uint32_t *warps_per_cta);

/* dg_search_batch for callers that cannot have device memory allocated for
 * them (hosts whose device memory belongs to a separate pool manager,
 * latency-critical threads that must not pay cudaMalloc's implicit device
 * synchronisation).  No counterpart in the reference: it is an addition of
 * this library.  It allocates nothing: its scratch (the search's work counter
 * and copies of the filter programs and per-query beams) lives in a
 * file-scope device array of 256 KiB that every GPU loading the library keeps
 * until the process exits.  Requires DG_FLAG_DEVICE_PTRS: queries and outputs
 * are device memory.  The filter programs (filter_ops, filter_offsets,
 * filter_pool) and per_query_beam stay HOST memory, as in dg_search_batch:
 * they are validated on the host and copied into the array with
 * cudaMemcpyAsync on the call's stream, so pinned arrays must stay valid
 * until the stream has passed the call.  Returns after enqueueing.  Per-call
 * parameters larger than the array (about 10k filter ops or 60k per-query
 * beams) are rejected with DG_EINVAL.  The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  Each device has its own copy of the array:
 * calls that overlap on the same device (any stream, any handle) share it
 * and race, so order them on one stream or wait between them; calls on
 * different devices do not interact.  Like dg_search_batch, the call records
 * its completion on one of the index's 16 completion events (blocking while
 * all 16 are in flight), so later row, adjacency, label and tombstone
 * updates and dg_index_destroy wait for it.  out_stats is not written. */
DG_API DgStatus dg_search_batch_static(DgIndex *idx, const DgSearchParams *p, const float *queries,
                                       uint32_t nq, uint32_t *out_ids, float *out_dists,
                                       uint32_t *out_counts);

/* FilteredDiskANN::count_matching (src/filtered.rs:508-510). */
DG_API DgStatus dg_count_matching(DgIndex *idx, const DgFilterOp *ops, uint32_t nops,
                           const uint64_t *pool, uint32_t pool_len, uint64_t *out_count);

/* ------------------------------------------------------------- serving loop */
/* Continuous batching over one DgIndex.  The reference serves a query as a
 * synchronous call (DiskANN::search_with_dists, src/lib.rs:683-714) and a
 * batch as a rayon par_iter over such calls (src/lib.rs:709-714); its benches
 * time sequential request loops (benches/benchmark.rs:183-207).  Here requests
 * are queued one at a time and a dispatcher thread forms batches of pending
 * requests with the same traversal, rerank size and filter presence (k, beam
 * and filter program stay per request, so one launch carries uneven k, beams
 * and filters), launching each batch on the next free stream slot.  Requests
 * that arrive while batches run are admitted as soon as a slot and memory
 * free up, and batches on different slots overlap on the device.  Memory is
 * admitted per batch: the server allocates one device arena (and a pinned
 * host arena) of hbm_budget_bytes at creation, and each batch takes a region
 * sized by its own queries, results at its largest k, beams and k; a batch
 * that does not fit is trimmed, and the dispatcher waits for regions of
 * batches in flight when not even one request fits.  A request returns
 * exactly what dg_search_batch returns for it alone. */
typedef struct DgServer DgServer;
typedef struct {
  uint32_t max_batch;        /* requests per launch */
  uint32_t streams;          /* batches in flight at once (one stream each) */
  uint32_t max_k;            /* largest k a request may ask for */
  uint32_t max_filter_ops;   /* largest filter program of one request */
  uint32_t max_wait_us;      /* how long a partial batch waits to fill; 0 = launch at once */
  uint64_t hbm_budget_bytes; /* the batch arena; 0 = room for a full batch at max_k on every stream.
                                creation fails with DG_ENOMEM when one request at max_k does not fit */
} DgServerConfig;
typedef struct {
  uint32_t k;
  uint32_t beam_width;
  uint32_t rerank_size;
  int32_t traversal; /* DgTraversal */
  const DgFilterOp *filter_ops; /* this request's postfix program (none = no filter) */
  uint32_t filter_nops;
  const uint64_t *filter_pool; /* IN values, offsets relative to this pool */
  uint32_t filter_pool_len;
} DgRequest;

DG_API DgStatus dg_server_create(DgIndex *idx, const DgServerConfig *cfg, DgServer **out);
/* Stops the dispatcher and waits for the batches in flight; call it after every
 * dg_server_wait has returned.  The index must outlive the server. */
DG_API DgStatus dg_server_destroy(DgServer *s);
/* Queues one request (query: f32[dim], copied); writes its ticket. */
DG_API DgStatus dg_server_submit(DgServer *s, const float *query, const DgRequest *req, uint64_t *ticket);
/* Waits at most timeout_us for a ticket; DG_ETIMEOUT leaves it pending for
 * another wait.  On success writes k ids / dists (padded past *out_count) and
 * the time from submission to completion, and releases the ticket. */
DG_API DgStatus dg_server_wait(DgServer *s, uint64_t ticket, int64_t timeout_us, uint32_t *out_ids,
                               float *out_dists, uint32_t *out_count, double *latency_us);
/* Batches launched, requests served, and the most batches ever in flight at once. */
DG_API DgStatus dg_server_stats(DgServer *s, uint64_t *batches, uint64_t *served, uint32_t *max_in_flight);
/* Replays an arrival trace: request i (query i, reqs[i]) is submitted by a
 * native thread at arrival_us[i] after the start.  Results go k-strided per
 * request into out_ids / out_dists (sum of reqs[i].k entries), counts into
 * out_counts, latencies into latency_us, and the time from the start until the
 * last result into *wall_us.  Waits at most timeout_us in total. */
DG_API DgStatus dg_server_run_trace(DgServer *s, const float *queries, uint32_t n, const DgRequest *reqs,
                                    const double *arrival_us, int64_t timeout_us, uint32_t *out_ids,
                                    float *out_dists, uint32_t *out_counts, double *latency_us,
                                    double *wall_us);

/* ------------------------------------------------------------------ SPFresh */
/* Posting lists of an SPFresh index (src/spfresh.rs:62-111,250-281): posting
 * slot b has a centroid, a live flag and block_len[b] entries (id, code) out
 * of block_cap; codes are the raw f32 vector (quantizer DG_Q_NONE), F16, int8,
 * PQ or RaBitQ residual codes against the posting centroid.  The raw store
 * holds every vector by id for the rerank.  Ids stay below 2^31. */
typedef struct DgSpfresh DgSpfresh;
typedef struct {
  uint32_t dim;
  int32_t metric;             /* DgMetric */
  int32_t device;
  uint32_t num_blocks;        /* posting slots, live or free */
  uint32_t block_cap;         /* entries per slot (2 * max_posting_size) */
  const float *centroids;     /* f32[num_blocks*dim] */
  const uint8_t *block_live;  /* u8[num_blocks] */
  const uint32_t *block_len;  /* u32[num_blocks] */
  const uint64_t *entry_ids;  /* u64[num_blocks*block_cap] */
  const uint8_t *entry_codes; /* [num_blocks*block_cap][code_size] */
  uint32_t code_size;         /* 4*dim raw, 2*dim F16, dim int8, M for PQ, padded/8+8 RaBitQ */
  int32_t quantizer;          /* DgQuantizer */
  uint32_t pq_M, pq_K;
  const float *pq_codebooks;  /* [M][K][dim/M] */
  float int8_scale, int8_offset;
  uint32_t rq_padded;
  const float *rq_signs;      /* f32[3*padded] */
  uint64_t id_capacity;       /* every id < id_capacity */
  uint64_t num_raw;           /* rows of `raw` given now (ids 0..num_raw-1) */
  const float *raw;           /* f32[num_raw*dim] */
  const uint8_t *deleted;     /* optional u8[id_capacity] tombstones */
} DgSpfreshDesc;

typedef struct {
  uint32_t k;
  uint32_t nprobe;      /* n_probe of SPFresh::search (src/spfresh.rs:886-895) */
  uint32_t rerank_size; /* SPFreshConfig::rerank_size (quantized postings) */
  float probe_ratio;    /* SPFreshConfig::probe_ratio (inf = off) */
  uint32_t flags;       /* DG_FLAG_* */
  void *stream;
} DgSpfreshParams;

/* SPFresh::build / open -> device-resident posting lists. */
DG_API DgStatus dg_spfresh_create(const DgSpfreshDesc *desc, DgSpfresh **out);
DG_API DgStatus dg_spfresh_destroy(DgSpfresh *s);
/* Replaces whole posting slots after host-side insert / split / merge
 * (Inner::rewrite / push, src/spfresh.rs:294-320): centroids f32[n*dim],
 * live u8[n], lens u32[n], ids u64[n*block_cap], codes [n*block_cap][code_size].
 * This call, dg_spfresh_put_raw and dg_spfresh_set_deleted run after every
 * search already issued on the handle has finished on the GPU (the reference
 * takes its RwLock for writing, src/spfresh.rs:862-871). */
DG_API DgStatus dg_spfresh_update_blocks(DgSpfresh *s, const uint32_t *blocks, uint32_t n,
                                         const float *centroids, const uint8_t *live,
                                         const uint32_t *lens, const uint64_t *entry_ids,
                                         const uint8_t *entry_codes);
/* Raw vectors of ids first_id .. first_id+n-1 (the raw store, src/spfresh.rs:283-286). */
DG_API DgStatus dg_spfresh_put_raw(DgSpfresh *s, uint64_t first_id, const float *vectors, uint64_t n);
/* SPFresh::delete tombstones (src/spfresh.rs:863-871); deleted = 0 clears. */
DG_API DgStatus dg_spfresh_set_deleted(DgSpfresh *s, const uint64_t *ids, uint64_t n, int32_t deleted);
/* The centroid and live flag of n posting slots, without their entries:
 * SPFresh's update path publishes new and freed postings with it before it
 * routes against them (Inner::new_posting / free_posting,
 * src/spfresh.rs:395-415).  centroids f32[n*dim], live u8[n]. */
DG_API DgStatus dg_spfresh_set_centroids(DgSpfresh *s, const uint32_t *blocks, uint32_t n, const float *centroids,
                                         const uint8_t *live);
/* Inner::nearest (src/spfresh.rs:358-378) for nv host vectors: the n (<= 64)
 * nearest live postings of each, ascending by (distance, slot), with every
 * distance summed in coordinate order in FP32 (brute force at every posting
 * count); rows are padded with DG_PAD / +inf past the live postings.  The
 * host update path routes its inserts, neighbourhoods and gc moves with it. */
DG_API DgStatus dg_spfresh_nearest(DgSpfresh *s, const float *vectors, uint32_t nv, uint32_t n,
                                   uint32_t *out_slots, float *out_dists);
/* SPFresh::search_with_dists / search_batch (src/spfresh.rs:671-770,886-908):
 * out_ids u64[nq*k] (DG_PAD64 padded), out_dists f32[nq*k], out_counts u32[nq].
 * Searches of one handle share its scratch: each waits on the GPU for the
 * previous one, whatever stream either runs on. */
DG_API DgStatus dg_spfresh_search_batch(DgSpfresh *s, const DgSpfreshParams *p, const float *queries,
                                        uint32_t nq, uint64_t *out_ids, float *out_dists,
                                        uint32_t *out_counts);

/* ---------------------------------------------------------- index building */
/* calculate_medoid (src/lib.rs:748-768) on the GPU. X is host f32[n*dim]. */
DG_API DgStatus dg_medoid(const float *X, uint64_t n, uint32_t dim, int32_t metric, int32_t device,
                   uint32_t *out_medoid);
/* build_vamana_graph (src/lib.rs:774-917) on the GPU: bootstrap, two
 * search+prune passes with symmetrisation, counter-based random draws from
 * `seed`.  X host f32[n*dim]; adjacency out host u32[n*R]. */
DG_API DgStatus dg_build_vamana(const float *X, uint64_t n, uint32_t dim, int32_t metric, uint32_t R,
                         uint32_t build_beam, float alpha, uint64_t seed, uint32_t medoid,
                         int32_t device, uint32_t *out_adjacency);
/* ProductQuantizer::train (src/pq.rs:51-119): Lloyd iterations on the GPU
 * from `seed`; codebooks out host f32[M*K*(dim/M)]. */
DG_API DgStatus dg_pq_train(const float *X, uint64_t n, uint32_t dim, uint32_t M, uint32_t K,
                     uint32_t iterations, uint64_t sample, uint64_t seed, int32_t device,
                     float *out_codebooks);
/* ProductQuantizer::encode (src/pq.rs:122-149) on the GPU. */
DG_API DgStatus dg_pq_encode(const float *X, uint64_t n, uint32_t dim, uint32_t M, uint32_t K,
                      const float *codebooks, int32_t device, uint8_t *out_codes);
/* RaBitQ::encode_with (src/rabitq.rs:218-256) on the GPU: codes of
 * padded/8+8 bytes of every row of X as residuals against `centroid`
 * (f32[dim]), with the quantizer's signs f32[3*padded].  SPFresh re-encodes
 * the entries of a posting against its new centroid with it
 * (Inner::encode, src/spfresh.rs:328-339). */
DG_API DgStatus dg_rabitq_encode(const float *X, uint64_t n, uint32_t dim, uint32_t padded, const float *centroid,
                                 const float *signs, int32_t device, uint8_t *out_codes);
/* The FP8 encoding of dg_index_enable_fp8 on the GPU: codes u8[n*dim] (e4m3)
 * and scales f32[n].  No counterpart in the reference. */
DG_API DgStatus dg_fp8_encode(const float *X, uint64_t n, uint32_t dim, int32_t device, uint8_t *out_codes,
                              float *out_scales);
/* Exact k nearest neighbours (brute force, FP64 accumulation) on the GPU. */
DG_API DgStatus dg_exact_knn(const float *X, uint64_t n, uint32_t dim, const float *Q, uint32_t nq,
                      uint32_t k, int32_t metric, int32_t device, uint32_t *out_ids,
                      float *out_dists);

DG_API const char *dg_last_error(void);
DG_API int32_t dg_version(void);

#ifdef __cplusplus
}
#endif
#endif
