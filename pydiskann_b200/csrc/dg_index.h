// dg_index.h -- the device-resident index behind a DgIndex handle.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <vector>

#include "dg_common.cuh"

struct DgIndex {
  int device = 0;
  uint64_t n = 0;
  uint32_t d = 0, dpad = 0, R = 0, medoid = 0;
  int32_t metric = DG_L2SQ;
  // HBM layout: every row starts on a 128-byte boundary when dpad*4 >= 128.
  float *vec = nullptr;       // [n][dpad] f32, zero padded
  uint16_t *bf16 = nullptr;   // [n][dpad] bf16 copy (optional)
  float *bf16_n2 = nullptr;   // [n] squared norms of the bf16 rows
  uint8_t *fp8 = nullptr;     // [n][dpad] e4m3 copy (optional)
  float2 *fp8_sn = nullptr;   // [n] (scale, |decoded|^2) of the e4m3 rows
  uint32_t *adj = nullptr;    // [n][R]
  int32_t quant = DG_Q_NONE;
  uint8_t *codes = nullptr;   // [n][code_stride]
  uint32_t code_size = 0, code_stride = 0;
  uint32_t pq_M = 0, pq_K = 0;
  float *pq_cb = nullptr;     // [M][K][d/M]
  float i8_scale = 1.0f, i8_offset = 0.0f;
  uint32_t *i8_norm = nullptr; // [n] sum of squared int8 codes (tensor-core L2)
  uint32_t *i8_sum = nullptr;  // [n] sum of int8 codes (tensor-core cosine / dot)
  uint32_t rq_padded = 0;
  float *rq_centroid = nullptr, *rq_signs = nullptr;
  float *dnorm2 = nullptr;    // [n] |decode(code)|^2 (cosine over PQ / RaBitQ codes)
  uint64_t *labels = nullptr; // [n][nf]
  uint32_t nf = 0;
  // base + delta (incremental) search state
  uint32_t seed2 = DG_PAD;             // second entry point, DG_PAD = none
  uint32_t *tomb = nullptr;            // [ceil(n/32)] deleted-id bitmap (device)
  std::vector<uint32_t> tomb_host;     // its host copy
  uint64_t ntomb = 0;                  // tombstone count the search config uses
  uint64_t code_limit = 0;             // rows >= code_limit have no codes (0 = every row has)
  // Launch schedule of a kind of search (traversal, working-set capacity,
  // filtered), chosen by dg_index_autotune: the visited-table size (log2 words
  // per query), the query order (0 = as given, 1 = grouped by nearest pivot),
  // the share of the resident CTAs per SM the grid uses (percent) and the
  // warps per CTA (4, 2 or 1: smaller CTAs pack an SM's shared memory more
  // finely when each query holds a large state).
  struct Schedule {
    uint32_t hbits = 0, order = 0, occ_pct = 100, wpb = 4;  // wpb: warps (queries in flight) per CTA
  };
  std::map<uint32_t, Schedule> tuned;
  bool forcing = false;   // the autotuner pins `force` while it times a candidate
  Schedule force{};
  uint32_t last_key = 0;  // key of the last search run while forcing
  Schedule last_tuned{};  // the schedule the last dg_index_autotune chose
  float *pivots = nullptr;  // [npiv][dpad] rows spread over the ids (query ordering)
  uint32_t npiv = 0;
  cudaStream_t stream = nullptr;
  uint64_t hbm_budget = 0, hbm_used = 0;
  std::mutex mu;
  // Per-call resources.  A call takes the next slot of a ring; a slot is reused
  // only after the event recorded at the end of its previous call completed,
  // so calls on different streams may overlap on the device.
  struct Buf {
    void *p = nullptr;
    size_t cap = 0;
  };
  struct Slot {
    Buf q, ids, dists, cnt, stats, fops, foffs, fpool, perl, perk, sched;
    uint32_t *counter = nullptr;  // work counters of the persistent grid (one per pipeline chunk)
    cudaEvent_t done = nullptr;
    bool pending = false;
  };
  static constexpr int kSlots = 16;
  Slot slots[kSlots];
  int next_slot = 0;
  // Host-pointer calls of many queries run as a pipeline of chunks: queries
  // in on pipe_in, kernels alternating on pipe_k[0..1] (a chunk's kernel
  // overlaps the previous one's tail), results out on pipe_out.  Created on
  // first use; calls on one handle are serialised, so one set suffices.
  static constexpr int kPipeChunks = 4;
  cudaStream_t pipe_in = nullptr, pipe_out = nullptr, pipe_k[2] = {nullptr, nullptr};
  cudaEvent_t pipe_start = nullptr, pipe_in_ev[kPipeChunks] = {}, pipe_k_ev[kPipeChunks] = {};
  std::vector<void *> allocations;
};

namespace dg {
uint32_t dpad_of(uint32_t d);
DgStatus dev_alloc(DgIndex *idx, void **p, size_t bytes);
DgStatus buf_reserve(DgIndex::Buf &b, size_t bytes);
// Sizes the per-call staging buffers of every call slot for batches of nq
// queries with `ops` filter instructions and `pool` IN values.
DgStatus reserve_call_buffers(DgIndex *idx, uint32_t nq, size_t ops, size_t pool);
// Query ordering by nearest pivot (dg_schedule.cu): pivots are set up once;
// order_queries writes perm[nq] (positions -> query ids) using bin[nq] and
// hist[npiv] as scratch.
uint32_t pivot_count(uint32_t dpad);
DgStatus ensure_pivots(DgIndex *idx);
DgStatus order_queries(const DgIndex *idx, const float *Q, uint32_t nq, uint32_t *perm, uint32_t *bin,
                       uint32_t *hist, cudaStream_t st);
DgStatus to_device(DgIndex *idx, void **dst, const void *src, size_t bytes);
// Rows of d floats from the host into [n][dpad] device rows, zero padded.
DgStatus upload_rows_f32(const float *host, uint64_t n, uint32_t d, uint32_t dpad, float *dev,
                         cudaStream_t st);
// Kernels used by the attach/encode entry points (dg_build.cu).
DgStatus encode_pq_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, uint32_t M,
                          uint32_t K, const float *cb, uint8_t *codes, uint32_t stride,
                          cudaStream_t st);
DgStatus encode_int8_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, float scale,
                            float offset, uint8_t *codes, uint32_t stride, cudaStream_t st);
DgStatus encode_f16_device(const float *vec, uint64_t n, uint32_t dpad, uint16_t *codes,
                           cudaStream_t st);
// BF16 rows (round to nearest even) and, when norms is not null, the squared
// norm of each BF16 row.
DgStatus encode_bf16_device(const float *vec, uint64_t n, uint32_t dpad, uint16_t *out,
                            cudaStream_t st, float *norms = nullptr);
DgStatus encode_rabitq_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, uint32_t P,
                              const float *centroid, const float *signs, uint8_t *codes,
                              uint32_t stride, cudaStream_t st);
// e4m3 rows with per-vector scales (and decoded squared norms) from f32 rows.
DgStatus encode_fp8_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, uint8_t *codes,
                           float2 *sn, cudaStream_t st);
// Sum of squared codes per vector for int8 codes.
// Per-row sum of squared codes (out) and, when sums is not null, sum of codes.
DgStatus int8_norms_device(const uint8_t *codes, uint64_t n, uint32_t stride, uint32_t *out, uint32_t *sums,
                           cudaStream_t st);
// |decode(code)|^2 per vector for PQ / RaBitQ codes (the cosine metric's |x|^2).
DgStatus decoded_norms_device(const DgIndex *idx, float *out, cudaStream_t st);
DgStatus count_matching_device(const uint64_t *labels, uint64_t n, uint32_t nf,
                               const DgFilterOp *ops, uint32_t nops, const uint64_t *pool,
                               unsigned long long *count, cudaStream_t st);
}  // namespace dg
