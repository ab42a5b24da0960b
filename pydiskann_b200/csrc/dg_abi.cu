// dg_abi.cu -- the extern "C" surface of libdgann (declared in include/dgann.h).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "dg_index.h"
#include "dg_launch.cuh"

namespace dg {

DgStatus dev_alloc(DgIndex *idx, void **p, size_t bytes) {
  if (idx->hbm_budget && idx->hbm_used + bytes > idx->hbm_budget)
    return fail(DG_ENOMEM, "index exceeds its HBM budget (" + std::to_string(idx->hbm_budget) + " bytes)");
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes ? bytes : 16);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  idx->hbm_used += bytes;
  idx->allocations.push_back(q);
  *p = q;
  return DG_OK;
}

// Grows geometrically (powers of two, at least 64 KiB): a reallocation
// synchronises the device, so a stream of varying batch sizes must not
// trigger one per call.
DgStatus buf_reserve(DgIndex::Buf &b, size_t bytes) {
  if (bytes <= b.cap) return DG_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = 64 * 1024;
  while (want < bytes) want *= 2;
  DG_CUDA(cudaMalloc(&b.p, want));
  b.cap = want;
  return DG_OK;
}

DgStatus to_device(DgIndex *idx, void **dst, const void *src, size_t bytes) {
  DgStatus s = dev_alloc(idx, dst, bytes);
  if (s != DG_OK) return s;
  DG_CUDA(cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, idx->stream));
  return DG_OK;
}

static int met_kind(int32_t metric) {
  return metric == DG_DOT ? MET_DOT : metric == DG_COSINE ? MET_COS : MET_L2;
}

// Lanes per row for a row of `chunks` 16-byte chunks.
static int lanes_per_row(uint32_t chunks) {
  if (chunks % 8 == 0) return 8;
  if (chunks % 4 == 0) return 4;
  return 2;
}

// Grows every call slot's staging buffers for per-call parameters to hold a
// batch of nq queries with `ops` filter instructions and `pool` IN values, so
// that later calls of that size reallocate nothing (a reallocation synchronises
// the device, a latency spike for every batch in flight), the scratch of a
// pivot-ordered launch included, and makes the pivot rows.  Waits for slots
// whose previous call is still running.
DgStatus reserve_call_buffers(DgIndex *idx, uint32_t nq, size_t ops, size_t pool) {
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  for (auto &sl : idx->slots) {
    if (sl.pending) {
      DG_CUDA(cudaEventSynchronize(sl.done));
      sl.pending = false;
    }
    DgStatus s;
    if ((s = buf_reserve(sl.fops, ops * sizeof(DgFilterOp))) != DG_OK) return s;
    if ((s = buf_reserve(sl.foffs, ((size_t)nq + 1) * 4)) != DG_OK) return s;
    if ((s = buf_reserve(sl.fpool, pool * 8)) != DG_OK) return s;
    if ((s = buf_reserve(sl.perl, (size_t)nq * 4)) != DG_OK) return s;
    if ((s = buf_reserve(sl.perk, (size_t)nq * 4)) != DG_OK) return s;
    // query-order scratch (a schedule that groups queries by nearest pivot)
    if ((s = buf_reserve(sl.sched, ((size_t)2 * nq + (size_t)DgIndex::kPipeChunks * pivot_count(idx->dpad)) * 4)) !=
        DG_OK)
      return s;
  }
  // the pivot rows of that order, copied once
  if ((size_t)pivot_count(idx->dpad) * idx->d * 4 <= 48 * 1024) return ensure_pivots(idx);
  return DG_OK;
}

}  // namespace dg

using namespace dg;

extern "C" {

DgStatus dg_index_create(const DgIndexDesc *desc, DgIndex **out) {
  if (!desc || !out) return fail(DG_EINVAL, "null argument");
  *out = nullptr;
  if (desc->dim == 0 || desc->num_vectors == 0)
    return fail(DG_EINVAL, "index needs at least one vector of dimension >= 1");
  if (desc->num_vectors >= (1ull << 31)) return fail(DG_EINVAL, "num_vectors must be < 2^31");
  if (desc->max_degree == 0 || desc->max_degree > (uint32_t)kStageCap)
    return fail(DG_EINVAL, "max_degree must be in [1, 256]");
  if (desc->medoid >= desc->num_vectors) return fail(DG_EINVAL, "medoid out of range");
  if (desc->metric < DG_L2SQ || desc->metric > DG_DOT) return fail(DG_EINVAL, "unknown metric");
  if (!desc->vectors || !desc->adjacency) return fail(DG_EINVAL, "vectors and adjacency are required");
  DG_CUDA(cudaSetDevice(desc->device));
  DgIndex *idx = new (std::nothrow) DgIndex();
  if (!idx) return fail(DG_ENOMEM, "host allocation failed");
  idx->device = desc->device;
  idx->n = desc->num_vectors;
  idx->d = desc->dim;
  idx->dpad = dpad_of(desc->dim);
  idx->R = desc->max_degree;
  idx->medoid = desc->medoid;
  idx->metric = desc->metric;
  idx->hbm_budget = desc->hbm_budget_bytes;
  DgStatus s = DG_OK;
  auto bail = [&](DgStatus st) {
    dg_index_destroy(idx);
    return st;
  };
  if (cudaStreamCreateWithFlags(&idx->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(DG_EDEVICE, "stream creation failed"));
  if ((s = dev_alloc(idx, (void **)&idx->vec, idx->n * idx->dpad * 4)) != DG_OK) return bail(s);
  if ((s = upload_rows_f32(desc->vectors, idx->n, idx->d, idx->dpad, idx->vec, idx->stream)) != DG_OK)
    return bail(s);
  if ((s = to_device(idx, (void **)&idx->adj, desc->adjacency, idx->n * idx->R * 4)) != DG_OK) return bail(s);
  for (auto &sl : idx->slots) {
    if (cudaMalloc(&sl.counter, 4 * DgIndex::kPipeChunks) != cudaSuccess)
      return bail(fail(DG_ENOMEM, "counter allocation"));
    if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
      return bail(fail(DG_EDEVICE, "event creation"));
  }
  if (cudaStreamSynchronize(idx->stream) != cudaSuccess) return bail(fail(DG_EDEVICE, "upload failed"));
  *out = idx;
  return DG_OK;
}

DgStatus dg_index_destroy(DgIndex *idx) {
  if (!idx) return DG_OK;
  cudaSetDevice(idx->device);
  if (idx->stream) cudaStreamSynchronize(idx->stream);
  for (auto &sl : idx->slots) {
    if (sl.done) {
      cudaEventSynchronize(sl.done);
      cudaEventDestroy(sl.done);
    }
    for (DgIndex::Buf *b : {&sl.q, &sl.ids, &sl.dists, &sl.cnt, &sl.stats, &sl.fops, &sl.foffs,
                            &sl.fpool, &sl.perl, &sl.perk})
      if (b->p) cudaFree(b->p);
    if (sl.counter) cudaFree(sl.counter);
  }
  for (void *p : idx->allocations) cudaFree(p);
  if (idx->stream) cudaStreamDestroy(idx->stream);
  for (cudaStream_t t : {idx->pipe_in, idx->pipe_out, idx->pipe_k[0], idx->pipe_k[1]})
    if (t) cudaStreamDestroy(t);
  if (idx->pipe_start) cudaEventDestroy(idx->pipe_start);
  for (int c = 0; c < DgIndex::kPipeChunks; ++c) {
    if (idx->pipe_in_ev[c]) cudaEventDestroy(idx->pipe_in_ev[c]);
    if (idx->pipe_k_ev[c]) cudaEventDestroy(idx->pipe_k_ev[c]);
  }
  delete idx;
  return DG_OK;
}

DgStatus dg_index_enable_bf16(DgIndex *idx) {
  if (!idx) return fail(DG_EINVAL, "null index");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  if (idx->bf16) return DG_OK;
  DgStatus s = dev_alloc(idx, (void **)&idx->bf16, idx->n * idx->dpad * 2);
  if (s != DG_OK) return s;
  if ((s = dev_alloc(idx, (void **)&idx->bf16_n2, idx->n * 4)) != DG_OK) return s;
  if ((s = encode_bf16_device(idx->vec, idx->n, idx->dpad, idx->bf16, idx->stream, idx->bf16_n2)) != DG_OK)
    return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_enable_fp8(DgIndex *idx) {
  if (!idx) return fail(DG_EINVAL, "null index");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  if (idx->fp8) return DG_OK;
  DgStatus s = dev_alloc(idx, (void **)&idx->fp8, idx->n * idx->dpad);
  if (s != DG_OK) return s;
  if ((s = dev_alloc(idx, (void **)&idx->fp8_sn, idx->n * sizeof(float2))) != DG_OK) return s;
  if ((s = encode_fp8_device(idx->vec, idx->n, idx->d, idx->dpad, idx->fp8, idx->fp8_sn, idx->stream)) != DG_OK)
    return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

static DgStatus attach_codes_common(DgIndex *idx, int quant, uint32_t code_size) {
  if (idx->quant != DG_Q_NONE) return fail(DG_EINVAL, "a quantizer is already attached");
  idx->quant = quant;
  idx->code_size = code_size;
  idx->code_stride = (code_size + 15u) & ~15u;
  DgStatus s = dev_alloc(idx, (void **)&idx->codes, idx->n * idx->code_stride);
  if (s != DG_OK) return s;
  DG_CUDA(cudaMemsetAsync(idx->codes, 0, idx->n * idx->code_stride, idx->stream));
  return DG_OK;
}

// Cosine over PQ / RaBitQ codes compares against the decoded code
// (src/quantized.rs:28-36); its squared norm is per vector, computed once.
static DgStatus attach_decoded_norms(DgIndex *idx) {
  if (idx->metric != DG_COSINE) return DG_OK;
  DgStatus s = dev_alloc(idx, (void **)&idx->dnorm2, idx->n * 4);
  if (s != DG_OK) return s;
  return decoded_norms_device(idx, idx->dnorm2, idx->stream);
}

static DgStatus upload_code_rows(DgIndex *idx, const uint8_t *codes) {
  DG_CUDA(cudaMemcpy2DAsync(idx->codes, idx->code_stride, codes, idx->code_size, idx->code_size,
                            idx->n, cudaMemcpyHostToDevice, idx->stream));
  return DG_OK;
}

DgStatus dg_index_attach_pq(DgIndex *idx, uint32_t M, uint32_t K, const float *codebooks,
                            const uint8_t *codes) {
  if (!idx || !codebooks) return fail(DG_EINVAL, "null argument");
  if (M == 0 || idx->d % M != 0)
    return fail(DG_EINVAL, "Dimension " + std::to_string(idx->d) + " not divisible by num_subspaces " +
                               std::to_string(M));
  if (K == 0 || K > 256) return fail(DG_EINVAL, "num_centroids must be in [1, 256] (codes are u8)");
  if (codes && K < 256) {  // every code indexes a K-entry table row
    for (uint64_t i = 0; i < idx->n * M; ++i)
      if (codes[i] >= K) return fail(DG_EINVAL, "PQ code " + std::to_string(codes[i]) + " >= num_centroids");
  }
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  DgStatus s = attach_codes_common(idx, DG_Q_PQ, M);
  if (s != DG_OK) return s;
  idx->pq_M = M;
  idx->pq_K = K;
  const size_t cbb = (size_t)M * K * (idx->d / M) * 4;
  if ((s = to_device(idx, (void **)&idx->pq_cb, codebooks, cbb)) != DG_OK) return s;
  if (codes) s = upload_code_rows(idx, codes);
  else s = encode_pq_device(idx->vec, idx->n, idx->d, idx->dpad, M, K, idx->pq_cb, idx->codes,
                            idx->code_stride, idx->stream);
  if (s != DG_OK) return s;
  if ((s = attach_decoded_norms(idx)) != DG_OK) return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_attach_int8(DgIndex *idx, float scale, float offset, const uint8_t *codes) {
  if (!idx) return fail(DG_EINVAL, "null index");
  if (!(scale > 0.0f)) return fail(DG_EINVAL, "int8 scale must be positive");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  DgStatus s = attach_codes_common(idx, DG_Q_INT8, idx->dpad);
  if (s != DG_OK) return s;
  idx->code_size = idx->d;
  idx->i8_scale = scale;
  idx->i8_offset = offset;
  if (codes) s = upload_code_rows(idx, codes);
  else s = encode_int8_device(idx->vec, idx->n, idx->d, idx->dpad, scale, offset, idx->codes,
                              idx->code_stride, idx->stream);
  if (s != DG_OK) return s;
  if ((s = dev_alloc(idx, (void **)&idx->i8_norm, idx->n * 4)) != DG_OK) return s;
  const bool decoded = idx->metric == DG_COSINE || idx->metric == DG_DOT;
  if (decoded && (s = dev_alloc(idx, (void **)&idx->i8_sum, idx->n * 4)) != DG_OK) return s;
  if ((s = int8_norms_device(idx->codes, idx->n, idx->code_stride, idx->i8_norm, idx->i8_sum, idx->stream)) !=
      DG_OK)
    return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_attach_f16(DgIndex *idx) { return dg_index_attach_f16_codes(idx, nullptr); }

DgStatus dg_index_attach_f16_codes(DgIndex *idx, const uint8_t *codes) {
  if (!idx) return fail(DG_EINVAL, "null index");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  DgStatus s = attach_codes_common(idx, DG_Q_F16, idx->dpad * 2);
  if (s != DG_OK) return s;
  idx->code_size = idx->d * 2;
  if (codes) s = upload_code_rows(idx, codes);
  else s = encode_f16_device(idx->vec, idx->n, idx->dpad, (uint16_t *)idx->codes, idx->stream);
  if (s != DG_OK) return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_attach_rabitq(DgIndex *idx, uint32_t padded, const float *centroid,
                                const float *signs, const uint8_t *codes) {
  if (!idx || !centroid || !signs) return fail(DG_EINVAL, "null argument");
  uint32_t want = 1;
  while (want < std::max(idx->d, 64u)) want <<= 1;
  if (padded != want) return fail(DG_EINVAL, "RaBitQ padded dim must be next_pow2(max(dim, 64))");
  if (padded > 4096) return fail(DG_ENOTSUP, "RaBitQ padded dim above 4096");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  DgStatus s = attach_codes_common(idx, DG_Q_RABITQ, padded / 8 + 8);
  if (s != DG_OK) return s;
  idx->rq_padded = padded;
  if ((s = to_device(idx, (void **)&idx->rq_centroid, centroid, idx->d * 4)) != DG_OK) return s;
  if ((s = to_device(idx, (void **)&idx->rq_signs, signs, 3ull * padded * 4)) != DG_OK) return s;
  if (codes) s = upload_code_rows(idx, codes);
  else s = encode_rabitq_device(idx->vec, idx->n, idx->d, idx->dpad, padded, idx->rq_centroid,
                                idx->rq_signs, idx->codes, idx->code_stride, idx->stream);
  if (s != DG_OK) return s;
  if ((s = attach_decoded_norms(idx)) != DG_OK) return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_attach_labels(DgIndex *idx, uint32_t num_fields, const uint64_t *labels) {
  if (!idx || (!labels && num_fields)) return fail(DG_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  if (idx->labels) return fail(DG_EINVAL, "labels are already attached");
  idx->nf = num_fields;
  DgStatus s = to_device(idx, (void **)&idx->labels, labels ? (const void *)labels : (const void *)"",
                         std::max<size_t>(idx->n * num_fields * 8, 8));
  if (s != DG_OK) return s;
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_set_entry_points(DgIndex *idx, const uint32_t *ids, uint32_t n) {
  if (!idx || !ids) return fail(DG_EINVAL, "null argument");
  if (n < 1 || n > 2) return fail(DG_EINVAL, "one or two entry points");
  for (uint32_t i = 0; i < n; ++i)
    if (ids[i] >= idx->n) return fail(DG_EINVAL, "entry point " + std::to_string(ids[i]) + " out of range");
  std::lock_guard<std::mutex> lk(idx->mu);
  idx->medoid = ids[0];
  idx->seed2 = n == 2 ? ids[1] : DG_PAD;
  return DG_OK;
}

// Orders idx->stream after every search already issued, on any stream (the
// reference's searches hold a read lock for their whole run, so an update
// never lands under one): rows, adjacency, labels and tombstones are rewritten
// only once those searches are done.  The caller holds idx->mu.
static cudaError_t after_searches(DgIndex *idx) {
  for (auto &sl : idx->slots) {
    if (!sl.pending) continue;
    const cudaError_t e = cudaStreamWaitEvent(idx->stream, sl.done, 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

DgStatus dg_index_set_tombstones(DgIndex *idx, const uint32_t *ids, uint64_t n, int32_t deleted,
                                 uint64_t tombstone_count) {
  if (!idx || (!ids && n)) return fail(DG_EINVAL, "null argument");
  for (uint64_t i = 0; i < n; ++i)
    if (ids[i] >= idx->n) return fail(DG_EINVAL, "tombstone id " + std::to_string(ids[i]) + " out of range");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  const size_t words = (idx->n + 31) / 32;
  if (!idx->tomb) {
    DgStatus s = dev_alloc(idx, (void **)&idx->tomb, words * 4);
    if (s != DG_OK) return s;
    idx->tomb_host.assign(words, 0u);
  }
  for (uint64_t i = 0; i < n; ++i) {
    const uint32_t bit = 1u << (ids[i] & 31);
    if (deleted) idx->tomb_host[ids[i] >> 5] |= bit;
    else idx->tomb_host[ids[i] >> 5] &= ~bit;
  }
  idx->ntomb = tombstone_count;
  DG_CUDA(after_searches(idx));
  DG_CUDA(cudaMemcpyAsync(idx->tomb, idx->tomb_host.data(), words * 4, cudaMemcpyHostToDevice, idx->stream));
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_set_code_limit(DgIndex *idx, uint64_t limit) {
  if (!idx) return fail(DG_EINVAL, "null index");
  if (limit > idx->n) return fail(DG_EINVAL, "code limit above the number of rows");
  std::lock_guard<std::mutex> lk(idx->mu);
  idx->code_limit = limit;
  return DG_OK;
}

DgStatus dg_index_update_rows(DgIndex *idx, uint64_t first, uint64_t count, const float *vectors,
                              const uint32_t *adjacency, const uint64_t *labels) {
  if (!idx) return fail(DG_EINVAL, "null index");
  if (first > idx->n || count > idx->n - first) return fail(DG_EINVAL, "rows out of range");
  const uint64_t coded = idx->code_limit && idx->code_limit < idx->n ? idx->code_limit : idx->n;
  if (vectors && idx->quant != DG_Q_NONE && first < coded)
    return fail(DG_ENOTSUP, "rows with quantized codes cannot be replaced (set a code limit below them)");
  if (labels && !idx->labels) return fail(DG_EINVAL, "the index has no labels");
  if (adjacency)
    for (uint64_t i = 0; i < count * idx->R; ++i)
      if (adjacency[i] != DG_PAD && adjacency[i] >= idx->n)
        return fail(DG_EINVAL, "neighbour id " + std::to_string(adjacency[i]) + " out of range");
  if (!count) return DG_OK;
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  DG_CUDA(after_searches(idx));
  DgStatus s;
  if (vectors) {
    float *rows = idx->vec + first * idx->dpad;
    if ((s = upload_rows_f32(vectors, count, idx->d, idx->dpad, rows, idx->stream)) != DG_OK) return s;
    if (idx->bf16 && (s = encode_bf16_device(rows, count, idx->dpad, idx->bf16 + first * idx->dpad, idx->stream,
                                             idx->bf16_n2 + first)) != DG_OK)
      return s;
    if (idx->fp8 && (s = encode_fp8_device(rows, count, idx->d, idx->dpad, idx->fp8 + first * idx->dpad,
                                           idx->fp8_sn + first, idx->stream)) != DG_OK)
      return s;
  }
  if (adjacency)
    DG_CUDA(cudaMemcpyAsync(idx->adj + first * idx->R, adjacency, count * idx->R * 4, cudaMemcpyHostToDevice,
                            idx->stream));
  if (labels)
    DG_CUDA(cudaMemcpyAsync(idx->labels + first * idx->nf, labels, count * idx->nf * 8, cudaMemcpyHostToDevice,
                            idx->stream));
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

DgStatus dg_index_get_codes(DgIndex *idx, uint8_t *out, uint64_t out_len, uint32_t *code_size) {
  if (!idx) return fail(DG_EINVAL, "null index");
  std::lock_guard<std::mutex> lk(idx->mu);
  if (idx->quant == DG_Q_NONE) return fail(DG_EINVAL, "no quantizer is attached");
  if (code_size) *code_size = idx->code_size;
  if (!out) return DG_OK;
  if (out_len < idx->n * (uint64_t)idx->code_size) return fail(DG_EINVAL, "output buffer smaller than n * code_size");
  DG_CUDA(cudaSetDevice(idx->device));
  DG_CUDA(cudaMemcpy2DAsync(out, idx->code_size, idx->codes, idx->code_stride, idx->code_size, idx->n,
                            cudaMemcpyDeviceToHost, idx->stream));
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  return DG_OK;
}

// Working-set entries a search needs (the kernel sizes w from the same rules)
// and whether it runs the filtered kernel: label filters (src/filtered.rs:35-56)
// or the tombstones of a base + delta index (tombstone_config,
// src/incremental.rs:505-516).
static uint64_t working_need(const DgIndex *idx, uint32_t maxL, uint32_t k, uint32_t search_k, bool any_filter,
                             bool *filt) {
  const bool tombed = idx->tomb && idx->ntomb > 0;
  uint64_t need = maxL;
  if (any_filter) need = std::max<uint64_t>({(uint64_t)maxL * 4, (uint64_t)k * 10, search_k});
  else if (tombed)
    need = std::max<uint64_t>({(uint64_t)maxL * 2, search_k + std::min<uint64_t>(idx->ntomb, maxL), search_k});
  // two entry points run in the general kernel (the 64-entry register-list
  // kernel seeds the medoid only), which a capacity above 64 selects
  if (idx->seed2 != DG_PAD) need = std::max<uint64_t>(need, 65);
  *filt = any_filter || tombed;
  return need;
}

// visited-table sizes dg_index_autotune tries (log2 words per query)
static constexpr uint32_t kTuneMinBits = 8, kTuneMaxBits = 13;

static uint32_t tune_key(int trav, int lcap, bool filt) {
  return ((uint32_t)trav << 20) | ((uint32_t)lcap << 1) | (filt ? 1u : 0u);
}

// The launch schedule of this kind of search: the autotuner's choice, or the
// defaults (a visited table sized by the beam, queries as given, every
// resident CTA); DG_HBITS, DG_ORDER and DG_OCC_PCT override each axis.
static DgIndex::Schedule schedule_of(DgIndex *idx, int trav, int lcap, bool filt, uint32_t maxL) {
  DgIndex::Schedule sc;
  sc.hbits = maxL <= 64 ? 10 : maxL <= 128 ? 11 : 12;
  {
    std::lock_guard<std::mutex> lk(idx->mu);
    if (idx->forcing) {
      sc = idx->force;
      idx->last_key = tune_key(trav, lcap, filt);
    } else {
      auto it = idx->tuned.find(tune_key(trav, lcap, filt));
      if (it != idx->tuned.end()) sc = it->second;
    }
  }
  if (const char *e = std::getenv("DG_HBITS")) sc.hbits = (uint32_t)std::max(6, std::min(14, atoi(e)));
  if (const char *e = std::getenv("DG_ORDER")) sc.order = atoi(e) != 0;
  if (const char *e = std::getenv("DG_OCC_PCT")) sc.occ_pct = (uint32_t)std::max(1, std::min(100, atoi(e)));
  if (const char *e = std::getenv("DG_WPB")) sc.wpb = atoi(e) == 1 ? 1u : atoi(e) == 2 ? 2u : 4u;
  return sc;
}

static uint32_t visited_bits(DgIndex *idx, int trav, int lcap, bool filt, uint32_t maxL) {
  return schedule_of(idx, trav, lcap, filt, maxL).hbits;
}

static void index_state(const DgIndex *idx, SearchArgs &a) {
  a.seed2 = idx->seed2;
  const bool tombed = idx->tomb && idx->ntomb > 0;
  a.tomb = tombed ? idx->tomb : nullptr;
  a.ntomb = tombed ? (uint32_t)std::min<uint64_t>(idx->ntomb, 0xffffffffu) : 0;
  a.code_limit = idx->code_limit && idx->code_limit < idx->n ? idx->code_limit : idx->n;
}

// Stack depth a postfix program needs; -1 if it is malformed.
static int program_depth(const DgFilterOp *ops, uint32_t n, uint64_t pool_len) {
  int sp = 0, mx = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const DgFilterOp &o = ops[i];
    if (o.op > DG_F_OR) return -1;
    if (o.op == DG_F_AND || o.op == DG_F_OR) {
      if ((int)o.field > sp) return -1;
      sp -= (int)o.field;
    } else if (o.op == DG_F_IN && (o.a > pool_len || o.b > pool_len - o.a)) {
      return -1;
    }
    ++sp;
    mx = std::max(mx, sp);
  }
  if (n > 0 && sp != 1) return -1;
  return mx;
}

// A slot whose previous call has finished on the device (the lowest such, so a
// caller that waits for each call keeps reusing the same buffers); when all
// are in flight, the next one of the ring after its call completes.
static cudaError_t take_slot(DgIndex *idx, DgIndex::Slot **out) {
  for (int i = 0; i < DgIndex::kSlots; ++i) {
    DgIndex::Slot &c = idx->slots[i];
    if (c.pending) {
      const cudaError_t e = cudaEventQuery(c.done);
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess) return e;
      c.pending = false;
    }
    *out = &c;
    return cudaSuccess;
  }
  DgIndex::Slot &c = idx->slots[idx->next_slot];
  idx->next_slot = (idx->next_slot + 1) % DgIndex::kSlots;
  const cudaError_t e = cudaEventSynchronize(c.done);
  if (e != cudaSuccess) return e;
  c.pending = false;
  *out = &c;
  return cudaSuccess;
}

static DgStatus pipe_init(DgIndex *idx) {
  if (idx->pipe_in) return DG_OK;
  for (cudaStream_t *t : {&idx->pipe_in, &idx->pipe_out, &idx->pipe_k[0], &idx->pipe_k[1]})
    DG_CUDA(cudaStreamCreateWithFlags(t, cudaStreamNonBlocking));
  DG_CUDA(cudaEventCreateWithFlags(&idx->pipe_start, cudaEventDisableTiming));
  for (int c = 0; c < DgIndex::kPipeChunks; ++c) {
    DG_CUDA(cudaEventCreateWithFlags(&idx->pipe_in_ev[c], cudaEventDisableTiming));
    DG_CUDA(cudaEventCreateWithFlags(&idx->pipe_k_ev[c], cudaEventDisableTiming));
  }
  return DG_OK;
}

static DgStatus stage_copy(DgIndex::Buf &b, const void *src, size_t bytes, cudaStream_t st) {
  DgStatus s = buf_reserve(b, bytes);
  if (s != DG_OK) return s;
  if (bytes) DG_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, st));
  return DG_OK;
}

DgStatus dg_search_batch(DgIndex *idx, const DgSearchParams *p, const float *queries, uint32_t nq,
                         uint32_t *out_ids, float *out_dists, uint32_t *out_counts,
                         uint32_t *out_stats) {
  if (!idx || !p) return fail(DG_EINVAL, "null argument");
  if (nq == 0) return DG_OK;
  if (!queries || !out_ids || !out_dists || !out_counts) return fail(DG_EINVAL, "null buffer");
  if (p->k == 0) return fail(DG_EINVAL, "k must be >= 1");
  const bool devptr = (p->flags & DG_FLAG_DEVICE_PTRS) != 0;
  // traversal kind
  int trav;
  switch (p->traversal) {
    case DG_TRAVERSE_F32: trav = TRAV_F32; break;
    case DG_TRAVERSE_BF16:
      if (!idx->bf16) return fail(DG_EINVAL, "BF16 traversal needs dg_index_enable_bf16");
      trav = TRAV_BF16;
      break;
    case DG_TRAVERSE_FP8:
      if (!idx->fp8) return fail(DG_EINVAL, "FP8 traversal needs dg_index_enable_fp8");
      trav = TRAV_FP8;
      break;
    case DG_TRAVERSE_CODES:
      switch (idx->quant) {
        case DG_Q_PQ: trav = TRAV_PQ; break;
        case DG_Q_INT8: trav = TRAV_INT8; break;
        case DG_Q_RABITQ: trav = TRAV_RABITQ; break;
        case DG_Q_F16: trav = TRAV_F16; break;
        default: return fail(DG_EINVAL, "code traversal needs an attached quantizer");
      }
      break;
    default: return fail(DG_EINVAL, "unknown traversal");
  }
  // per-query beams and filters
  uint32_t maxL = p->beam_width;
  if (p->per_query_beam) {
    maxL = 0;
    for (uint32_t i = 0; i < nq; ++i) maxL = std::max(maxL, p->per_query_beam[i]);
    for (uint32_t i = 0; i < nq; ++i)
      if (p->per_query_beam[i] == 0) return fail(DG_EINVAL, "beam_width must be >= 1");
  }
  if (maxL == 0) return fail(DG_EINVAL, "beam_width must be >= 1");
  if (p->per_query_k)
    for (uint32_t i = 0; i < nq; ++i)
      if (p->per_query_k[i] == 0 || p->per_query_k[i] > p->k)
        return fail(DG_EINVAL, "per_query_k must be in [1, k]");
  const uint32_t total_ops = p->filter_offsets ? p->filter_offsets[nq] : p->filter_nops;
  bool any_filter = false;
  if (p->filter_offsets) {
    if (p->filter_offsets[0] != 0) return fail(DG_EINVAL, "filter_offsets[0] must be 0");
    for (uint32_t i = 0; i < nq; ++i) {
      if (p->filter_offsets[i + 1] < p->filter_offsets[i]) return fail(DG_EINVAL, "filter_offsets not monotone");
      const uint32_t c = p->filter_offsets[i + 1] - p->filter_offsets[i];
      if (c) {
        any_filter = true;
        int dep = program_depth(p->filter_ops + p->filter_offsets[i], c, p->filter_pool_len);
        if (dep < 0 || dep > kFilterStack) return fail(DG_EINVAL, "malformed filter program");
      }
    }
  } else if (p->filter_nops) {
    any_filter = true;
    int dep = program_depth(p->filter_ops, p->filter_nops, p->filter_pool_len);
    if (dep < 0 || dep > kFilterStack) return fail(DG_EINVAL, "malformed filter program");
  }
  if (any_filter && !p->filter_ops) return fail(DG_EINVAL, "filter ops missing");
  if (any_filter && !idx->labels) return fail(DG_EINVAL, "filtered search needs attached labels");
  const bool reranked = trav != TRAV_F32 && p->rerank_size > 0;
  const uint32_t search_k = reranked ? std::max(p->rerank_size, p->k) : p->k;
  bool filt = false;
  const uint64_t need = working_need(idx, maxL, p->k, search_k, any_filter, &filt);
  int lcap = need <= 64 ? 64 : need <= 256 ? 256 : need <= 1024 ? 1024 : 0;
  if (!lcap) return fail(DG_ENOTSUP, "beam width / expanded beam above 1024 is not supported");
  if (reranked && !filt && search_k > 1024) return fail(DG_ENOTSUP, "rerank size above 1024");
  // launch schedule: visited table of 2^hbits words as buckets of eight
  // 16-bit tags (about 3 tags per visited node at these beams), query order
  // and CTAs per SM, as dg_index_autotune measured fastest for this kind of
  // search (defaults otherwise); DG_HBITS overrides the table size
  const DgIndex::Schedule sched = schedule_of(idx, trav, lcap, filt, maxL);
  const uint32_t hbits = sched.hbits;
  uint32_t hB = 1;
  while (hB < 32 && (1ull << hB) < idx->n) ++hB;
  hB = std::max(hB, hbits);

  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  cudaStream_t st = (p->flags & DG_FLAG_STREAM) || p->stream ? (cudaStream_t)p->stream : idx->stream;
  DgIndex::Slot *slp = nullptr;
  DG_CUDA(take_slot(idx, &slp));
  DgIndex::Slot &sl = *slp;
  DgStatus s;
  SearchArgs a{};
  a.n = idx->n;
  a.d = idx->d;
  a.dpad = idx->dpad;
  a.R = idx->R;
  a.medoid = idx->medoid;
  index_state(idx, a);
  a.metric = idx->metric;
  a.vec_f32 = idx->vec;
  a.vec_bf16 = idx->bf16;
  a.bf16_n2 = idx->bf16_n2;
  a.adj = idx->adj;
  a.codes = idx->codes;
  a.code_stride = idx->code_stride;
  a.pq_M = idx->pq_M;
  a.pq_K = idx->pq_K;
  a.pq_ds = idx->pq_M ? idx->d / idx->pq_M : 0;
  a.pq_cb = idx->pq_cb;
  a.i8_scale = idx->i8_scale;
  a.i8_offset = idx->i8_offset;
  a.i8_norm = idx->i8_norm;
  a.i8_sum = idx->i8_sum;
  a.vec_fp8 = idx->fp8;
  a.fp8_sn = idx->fp8_sn;
  a.rq_padded = idx->rq_padded;
  a.rq_centroid = idx->rq_centroid;
  a.rq_signs = idx->rq_signs;
  a.dnorm2 = idx->dnorm2;
  a.labels = idx->labels;
  a.nf = idx->nf;
  a.nq = nq;
  a.k = p->k;
  a.L = p->beam_width;
  a.rerank = p->rerank_size;
  a.hbits = hbits;
  a.hB = hB;
  if (any_filter) {
    if ((s = stage_copy(sl.fops, p->filter_ops, (size_t)total_ops * sizeof(DgFilterOp), st)) != DG_OK) return s;
    a.fops = (const DgFilterOp *)sl.fops.p;
    a.fnops = p->filter_offsets ? 0 : p->filter_nops;
    if (p->filter_offsets) {
      if ((s = stage_copy(sl.foffs, p->filter_offsets, (size_t)(nq + 1) * 4, st)) != DG_OK) return s;
      a.foffs = (const uint32_t *)sl.foffs.p;
    }
    if ((s = stage_copy(sl.fpool, p->filter_pool, (size_t)p->filter_pool_len * 8, st)) != DG_OK) return s;
    a.fpool = (const uint64_t *)sl.fpool.p;
  }
  if (p->per_query_beam) {
    if ((s = stage_copy(sl.perl, p->per_query_beam, (size_t)nq * 4, st)) != DG_OK) return s;
    a.perL = (const uint32_t *)sl.perl.p;
  }
  if (p->per_query_k) {
    if ((s = stage_copy(sl.perk, p->per_query_k, (size_t)nq * 4, st)) != DG_OK) return s;
    a.perK = (const uint32_t *)sl.perk.p;
  }
  const size_t kq = (size_t)nq * p->k;
  // host calls of many queries: chunks whose copies overlap the other chunks' kernels
  uint32_t chunks = devptr || nq < 4096 ? 1u : std::min<uint32_t>(DgIndex::kPipeChunks, nq / 2048);
  if (const char *e = std::getenv("DG_PIPE_CHUNKS"); e && chunks > 1)  // override for measurements
    chunks = (uint32_t)std::max(1, std::min(DgIndex::kPipeChunks, atoi(e)));
  if (devptr) {
    a.Q = queries;
    a.out_ids = out_ids;
    a.out_d = out_dists;
    a.out_cnt = out_counts;
    a.out_stats = out_stats;
  } else {
    if (chunks > 1) {
      if ((s = buf_reserve(sl.q, (size_t)nq * idx->d * 4)) != DG_OK) return s;
    } else if ((s = stage_copy(sl.q, queries, (size_t)nq * idx->d * 4, st)) != DG_OK) {
      return s;
    }
    if ((s = buf_reserve(sl.ids, kq * 4)) != DG_OK) return s;
    if ((s = buf_reserve(sl.dists, kq * 4)) != DG_OK) return s;
    if ((s = buf_reserve(sl.cnt, (size_t)nq * 4)) != DG_OK) return s;
    a.Q = (const float *)sl.q.p;
    a.out_ids = (uint32_t *)sl.ids.p;
    a.out_d = (float *)sl.dists.p;
    a.out_cnt = (uint32_t *)sl.cnt.p;
    if (out_stats) {
      if ((s = buf_reserve(sl.stats, (size_t)nq * 8)) != DG_OK) return s;
      a.out_stats = (uint32_t *)sl.stats.p;
    }
  }
  a.counter = sl.counter;
  a.occ_pct = sched.occ_pct;
  a.wpb = sched.wpb;
  // query order: grouped by nearest pivot (per pipeline chunk) when the
  // schedule asks for it and the pivots fit the ordering kernel
  const bool ordered = sched.order && (size_t)pivot_count(idx->dpad) * idx->d * 4 <= 48 * 1024;
  // scratch: perm [nq] | pivot of each query [nq] | bin counts [pipeline chunk][npiv]
  uint32_t *perm = nullptr, *obin = nullptr, *ohist = nullptr;
  if (ordered) {
    if ((s = ensure_pivots(idx)) != DG_OK) return s;
    if ((s = buf_reserve(sl.sched, ((size_t)2 * nq + (size_t)DgIndex::kPipeChunks * idx->npiv) * 4)) != DG_OK)
      return s;
    perm = (uint32_t *)sl.sched.p;
    obin = perm + nq;
    ohist = obin + nq;
  }

  const int met = met_kind(idx->metric);
  int lpr = 1;
  if (trav == TRAV_F32) lpr = 8;
  else if (trav == TRAV_BF16 || trav == TRAV_F16) lpr = lanes_per_row(idx->dpad / 8);
  else if (trav == TRAV_INT8) lpr = lanes_per_row(idx->code_stride / 16);
  const WarpLayout Ly = warp_layout(trav, lcap, filt, hbits, idx->dpad, idx->pq_M, idx->pq_K,
                                    idx->rq_padded,
                                    (trav == TRAV_RABITQ || trav == TRAV_INT8) && met_kind(idx->metric) != MET_L2,
                                    idx->R, true);
  auto launch = [&](const SearchArgs &a0, cudaStream_t ss) -> DgStatus {
    LaunchInfo info;
    SearchArgs aa = a0;
    if (ordered) {  // positions of this launch's queries (relative to aa.Q); chunk c counts with counter c
      const size_t q0 = (size_t)(aa.Q - a.Q) / idx->d, c = (size_t)(aa.counter - a.counter);
      DgStatus so = order_queries(idx, aa.Q, aa.nq, perm + q0, obin + q0, ohist + c * idx->npiv, ss);
      if (so != DG_OK) return so;
      aa.perm = perm + q0;
    }
    DG_CUDA(cudaMemsetAsync(aa.counter, 0, 4, ss));
    switch (trav) {
      case TRAV_F32: return launch_search_f32(aa, Ly, met, lpr, lcap, filt, ss, &info);
      case TRAV_BF16: return launch_search_bf16(aa, Ly, met, lpr, lcap, filt, ss, &info);
      case TRAV_F16: return launch_search_f16(aa, Ly, met, lpr, lcap, filt, ss, &info);
      case TRAV_INT8: return launch_search_int8(aa, Ly, met, lpr, lcap, filt, ss, &info);
      case TRAV_PQ: return launch_search_pq(aa, Ly, met, lpr, lcap, filt, ss, &info);
      case TRAV_FP8: return launch_search_fp8(aa, Ly, met, lpr, lcap, filt, ss, &info);
      default: return launch_search_rabitq(aa, Ly, met, lpr, lcap, filt, ss, &info);
    }
  };
  if (chunks > 1) {
    if ((s = pipe_init(idx)) != DG_OK) return s;
    DG_CUDA(cudaEventRecord(idx->pipe_start, st));  // after the staged programs / beams on st
    for (cudaStream_t t : {idx->pipe_in, idx->pipe_out, idx->pipe_k[0], idx->pipe_k[1]})
      DG_CUDA(cudaStreamWaitEvent(t, idx->pipe_start, 0));
    const size_t d = idx->d, k = p->k;
    for (uint32_t c = 0; c < chunks; ++c) {
      const size_t q0 = (size_t)nq * c / chunks, q1 = (size_t)nq * (c + 1) / chunks;
      DG_CUDA(cudaMemcpyAsync((float *)sl.q.p + q0 * d, queries + q0 * d, (q1 - q0) * d * 4,
                              cudaMemcpyHostToDevice, idx->pipe_in));
      DG_CUDA(cudaEventRecord(idx->pipe_in_ev[c], idx->pipe_in));
    }
    for (uint32_t c = 0; c < chunks; ++c) {
      const size_t q0 = (size_t)nq * c / chunks, q1 = (size_t)nq * (c + 1) / chunks;
      SearchArgs ac = a;
      ac.Q = a.Q + q0 * d;
      ac.nq = (uint32_t)(q1 - q0);
      ac.out_ids = a.out_ids + q0 * k;
      ac.out_d = a.out_d + q0 * k;
      ac.out_cnt = a.out_cnt + q0;
      if (a.out_stats) ac.out_stats = a.out_stats + 2 * q0;
      if (a.perL) ac.perL = a.perL + q0;
      if (a.perK) ac.perK = a.perK + q0;
      if (a.foffs) ac.foffs = a.foffs + q0;
      ac.counter = sl.counter + c;
      cudaStream_t ks = idx->pipe_k[c & 1];
      DG_CUDA(cudaStreamWaitEvent(ks, idx->pipe_in_ev[c], 0));
      if ((s = launch(ac, ks)) != DG_OK) return s;
      DG_CUDA(cudaEventRecord(idx->pipe_k_ev[c], ks));
      DG_CUDA(cudaStreamWaitEvent(idx->pipe_out, idx->pipe_k_ev[c], 0));
      DG_CUDA(cudaMemcpyAsync(out_ids + q0 * k, ac.out_ids, (q1 - q0) * k * 4, cudaMemcpyDeviceToHost,
                              idx->pipe_out));
      DG_CUDA(cudaMemcpyAsync(out_dists + q0 * k, ac.out_d, (q1 - q0) * k * 4, cudaMemcpyDeviceToHost,
                              idx->pipe_out));
      DG_CUDA(cudaMemcpyAsync(out_counts + q0, ac.out_cnt, (q1 - q0) * 4, cudaMemcpyDeviceToHost, idx->pipe_out));
      if (out_stats)
        DG_CUDA(cudaMemcpyAsync(out_stats + 2 * q0, ac.out_stats, (q1 - q0) * 8, cudaMemcpyDeviceToHost,
                                idx->pipe_out));
    }
    DG_CUDA(cudaEventRecord(sl.done, idx->pipe_out));
    DG_CUDA(cudaStreamWaitEvent(st, sl.done, 0));  // later work on the caller's stream follows
    DG_CUDA(cudaEventSynchronize(sl.done));
    return DG_OK;
  }
  if ((s = launch(a, st)) != DG_OK) return s;
  if (!devptr) {
    DG_CUDA(cudaMemcpyAsync(out_ids, a.out_ids, kq * 4, cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaMemcpyAsync(out_dists, a.out_d, kq * 4, cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaMemcpyAsync(out_counts, a.out_cnt, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
    if (out_stats) DG_CUDA(cudaMemcpyAsync(out_stats, a.out_stats, (size_t)nq * 8, cudaMemcpyDeviceToHost, st));
  }
  DG_CUDA(cudaEventRecord(sl.done, st));
  sl.pending = true;
  if (!devptr) {
    DG_CUDA(cudaEventSynchronize(sl.done));
    sl.pending = false;
  }
  return DG_OK;
}

DgStatus dg_index_autotune(DgIndex *idx, const DgSearchParams *p, const float *queries, uint32_t nq,
                           uint32_t reps, uint32_t *best_hbits, float *ms_per_call) {
  if (!idx || !p || !queries || nq == 0) return fail(DG_EINVAL, "null argument or no queries");
  reps = std::max(reps, 1u);
  DG_CUDA(cudaSetDevice(idx->device));
  struct Scratch {
    void *p[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t e[2] = {nullptr, nullptr};
    ~Scratch() {
      if (st) cudaStreamSynchronize(st);
      for (void *q : p)
        if (q) cudaFree(q);
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
      if (st) cudaStreamDestroy(st);
    }
  } sc;
  const size_t kq = (size_t)nq * std::max(p->k, 1u);
  const float *dq = queries;
  if (!(p->flags & DG_FLAG_DEVICE_PTRS)) {
    DG_CUDA(cudaMalloc(&sc.p[0], (size_t)nq * idx->d * 4));
    DG_CUDA(cudaMemcpy(sc.p[0], queries, (size_t)nq * idx->d * 4, cudaMemcpyHostToDevice));
    dq = (const float *)sc.p[0];
  }
  DG_CUDA(cudaMalloc(&sc.p[1], kq * 4));
  DG_CUDA(cudaMalloc(&sc.p[2], kq * 4));
  DG_CUDA(cudaMalloc(&sc.p[3], (size_t)nq * 4));
  DG_CUDA(cudaStreamCreateWithFlags(&sc.st, cudaStreamNonBlocking));
  DG_CUDA(cudaEventCreate(&sc.e[0]));
  DG_CUDA(cudaEventCreate(&sc.e[1]));
  DgSearchParams pp = *p;
  pp.flags = p->flags | DG_FLAG_DEVICE_PTRS | DG_FLAG_STREAM;
  pp.stream = sc.st;
  auto run = [&]() {
    return dg_search_batch(idx, &pp, dq, nq, (uint32_t *)sc.p[1], (float *)sc.p[2], (uint32_t *)sc.p[3], nullptr);
  };
  // mean time per call of one schedule (a warm-up call first); DG_ENOTSUP when
  // it does not fit (a visited table too large for shared memory)
  auto time_schedule = [&](const DgIndex::Schedule &c, float *ms) -> DgStatus {
    {
      std::lock_guard<std::mutex> lk(idx->mu);
      idx->forcing = true;
      idx->force = c;
    }
    DgStatus s = run();
    if (s != DG_OK) return s;
    cudaEventRecord(sc.e[0], sc.st);
    for (uint32_t r = 0; r < reps && s == DG_OK; ++r) s = run();
    cudaEventRecord(sc.e[1], sc.st);
    if (s != DG_OK) return s;
    DG_CUDA(cudaEventSynchronize(sc.e[1]));
    DG_CUDA(cudaEventElapsedTime(ms, sc.e[0], sc.e[1]));
    *ms /= (float)reps;
    return DG_OK;
  };
  DgIndex::Schedule best{};
  float best_ms = 0.0f;
  bool have = false;
  uint32_t key = 0;
  DgStatus result = DG_OK;
  auto consider = [&](const DgIndex::Schedule &c, float *ms_out) -> DgStatus {
    float ms = 0.0f;
    const DgStatus s = time_schedule(c, &ms);
    if (s == DG_ENOTSUP) return DG_OK;
    if (s != DG_OK) return s;
    if (ms_out) *ms_out = ms;
    if (!have || ms < best_ms) {
      have = true;
      best = c;
      best_ms = ms;
      std::lock_guard<std::mutex> lk(idx->mu);
      key = idx->last_key;
    }
    return DG_OK;
  };
  // coordinate search: the visited-table size (queries as given, every
  // resident CTA), then the query order, then the CTAs per SM
  for (uint32_t hb = kTuneMinBits; hb <= kTuneMaxBits && result == DG_OK; ++hb) {
    if (ms_per_call) ms_per_call[hb - kTuneMinBits] = -1.0f;
    DgIndex::Schedule c;
    c.hbits = hb;
    result = consider(c, ms_per_call ? ms_per_call + (hb - kTuneMinBits) : nullptr);
  }
  if (result == DG_OK && have) {
    DgIndex::Schedule c = best;
    c.order = 1;
    result = consider(c, nullptr);
  }
  for (uint32_t pct : {75u, 50u}) {
    if (result != DG_OK || !have) break;
    DgIndex::Schedule c = best;
    c.occ_pct = pct;
    result = consider(c, nullptr);
  }
  for (uint32_t w : {2u, 1u}) {
    if (result != DG_OK || !have) break;
    DgIndex::Schedule c = best;
    c.wpb = w;
    result = consider(c, nullptr);
  }
  std::lock_guard<std::mutex> lk(idx->mu);
  idx->forcing = false;
  if (result != DG_OK) return result;
  if (!have) return fail(DG_ENOTSUP, "no visited-table size fits this search");
  idx->tuned[key] = best;
  idx->last_tuned = best;
  if (best_hbits) *best_hbits = best.hbits;
  return DG_OK;
}

DgStatus dg_index_tuned_schedule(DgIndex *idx, uint32_t *hbits, uint32_t *order, uint32_t *occ_pct,
                                 uint32_t *warps_per_cta) {
  if (!idx) return fail(DG_EINVAL, "null index");
  std::lock_guard<std::mutex> lk(idx->mu);
  if (hbits) *hbits = idx->last_tuned.hbits;
  if (order) *order = idx->last_tuned.order;
  if (occ_pct) *occ_pct = idx->last_tuned.occ_pct;
  if (warps_per_cta) *warps_per_cta = idx->last_tuned.wpb;
  return DG_OK;
}

DgStatus dg_count_matching(DgIndex *idx, const DgFilterOp *ops, uint32_t nops,
                           const uint64_t *pool, uint32_t pool_len, uint64_t *out_count) {
  if (!idx || !out_count) return fail(DG_EINVAL, "null argument");
  if (nops == 0) {
    *out_count = idx->n;
    return DG_OK;
  }
  if (!idx->labels) return fail(DG_EINVAL, "count_matching needs attached labels");
  int dep = program_depth(ops, nops, pool_len);
  if (dep < 0 || dep > kFilterStack) return fail(DG_EINVAL, "malformed filter program");
  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  DgIndex::Slot *slp = nullptr;
  DG_CUDA(take_slot(idx, &slp));
  DgIndex::Slot &sl = *slp;
  DgStatus s;
  if ((s = stage_copy(sl.fops, ops, (size_t)nops * sizeof(DgFilterOp), idx->stream)) != DG_OK) return s;
  if ((s = stage_copy(sl.fpool, pool, (size_t)pool_len * 8, idx->stream)) != DG_OK) return s;
  if ((s = buf_reserve(sl.cnt, 8)) != DG_OK) return s;
  DG_CUDA(cudaMemsetAsync(sl.cnt.p, 0, 8, idx->stream));
  if ((s = count_matching_device(idx->labels, idx->n, idx->nf, (const DgFilterOp *)sl.fops.p, nops,
                                 (const uint64_t *)sl.fpool.p, (unsigned long long *)sl.cnt.p,
                                 idx->stream)) != DG_OK)
    return s;
  unsigned long long c = 0;
  DG_CUDA(cudaMemcpyAsync(&c, sl.cnt.p, 8, cudaMemcpyDeviceToHost, idx->stream));
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  *out_count = c;
  return DG_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Search without any device allocation.
//
// Some callers cannot have device memory allocated on their behalf: hosts
// whose device memory is owned by a separate pool manager, and
// latency-critical request threads that must not pay cudaMalloc's implicit
// device-wide synchronisation.  dg_search_batch_static serves them: its only
// scratch memory (the work counter of the persistent grid and copies of the
// per-call filter programs and beams) lives in the file-scope array below,
// which every GPU that loads the library holds until the process exits.
namespace dg {

constexpr size_t kStaticScratchBytes = 256 * 1024;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_static_mu;
static void *g_static_addr[kMaxDevices];

// Device address of g_static_scratch on `device` (the current device).  In host
// code the array's name only stands in for the symbol, so the address is asked
// for once per device, with that device current, and kept.
static DgStatus static_scratch(int device, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (device < 0 || device >= kMaxDevices) return fail(DG_EINVAL, "device ordinal out of range");
  if (!g_static_addr[device]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
    g_static_addr[device] = ptr;
  }
  *out = static_cast<unsigned char *>(g_static_addr[device]);
  return DG_OK;
}

}  // namespace dg

extern "C" DgStatus dg_search_batch_static(DgIndex *idx, const DgSearchParams *p, const float *queries,
                                           uint32_t nq, uint32_t *out_ids, float *out_dists,
                                           uint32_t *out_counts) {
  if (!idx || !p) return fail(DG_EINVAL, "null argument");
  if (nq == 0) return DG_OK;
  if (!queries || !out_ids || !out_dists || !out_counts) return fail(DG_EINVAL, "null buffer");
  if (!(p->flags & DG_FLAG_DEVICE_PTRS))
    return fail(DG_EINVAL, "dg_search_batch_static needs device pointers (DG_FLAG_DEVICE_PTRS)");
  if (p->k == 0) return fail(DG_EINVAL, "k must be >= 1");
  int trav;
  switch (p->traversal) {
    case DG_TRAVERSE_F32: trav = TRAV_F32; break;
    case DG_TRAVERSE_BF16:
      if (!idx->bf16) return fail(DG_EINVAL, "BF16 traversal needs dg_index_enable_bf16");
      trav = TRAV_BF16;
      break;
    case DG_TRAVERSE_FP8:
      if (!idx->fp8) return fail(DG_EINVAL, "FP8 traversal needs dg_index_enable_fp8");
      trav = TRAV_FP8;
      break;
    case DG_TRAVERSE_CODES:
      switch (idx->quant) {
        case DG_Q_PQ: trav = TRAV_PQ; break;
        case DG_Q_INT8: trav = TRAV_INT8; break;
        case DG_Q_RABITQ: trav = TRAV_RABITQ; break;
        case DG_Q_F16: trav = TRAV_F16; break;
        default: return fail(DG_EINVAL, "code traversal needs an attached quantizer");
      }
      break;
    default: return fail(DG_EINVAL, "unknown traversal");
  }
  uint32_t maxL = p->beam_width;
  if (p->per_query_beam) {
    maxL = 0;
    for (uint32_t i = 0; i < nq; ++i) {
      if (p->per_query_beam[i] == 0) return fail(DG_EINVAL, "beam_width must be >= 1");
      maxL = std::max(maxL, p->per_query_beam[i]);
    }
  }
  if (maxL == 0) return fail(DG_EINVAL, "beam_width must be >= 1");
  if (p->per_query_k)
    for (uint32_t i = 0; i < nq; ++i)
      if (p->per_query_k[i] == 0 || p->per_query_k[i] > p->k)
        return fail(DG_EINVAL, "per_query_k must be in [1, k]");
  const uint32_t total_ops = p->filter_offsets ? p->filter_offsets[nq] : p->filter_nops;
  bool any_filter = false;
  if (p->filter_offsets) {
    if (p->filter_offsets[0] != 0) return fail(DG_EINVAL, "filter_offsets[0] must be 0");
    for (uint32_t i = 0; i < nq; ++i) {
      if (p->filter_offsets[i + 1] < p->filter_offsets[i]) return fail(DG_EINVAL, "filter_offsets not monotone");
      const uint32_t c = p->filter_offsets[i + 1] - p->filter_offsets[i];
      if (c) {
        any_filter = true;
        const int dep = program_depth(p->filter_ops + p->filter_offsets[i], c, p->filter_pool_len);
        if (dep < 0 || dep > kFilterStack) return fail(DG_EINVAL, "malformed filter program");
      }
    }
  } else if (p->filter_nops) {
    any_filter = true;
    const int dep = program_depth(p->filter_ops, p->filter_nops, p->filter_pool_len);
    if (dep < 0 || dep > kFilterStack) return fail(DG_EINVAL, "malformed filter program");
  }
  if (any_filter && !p->filter_ops) return fail(DG_EINVAL, "filter ops missing");
  if (any_filter && !idx->labels) return fail(DG_EINVAL, "filtered search needs attached labels");
  const bool reranked = trav != TRAV_F32 && p->rerank_size > 0;
  const uint32_t search_k = reranked ? std::max(p->rerank_size, p->k) : p->k;
  bool filt = false;
  const uint64_t need = working_need(idx, maxL, p->k, search_k, any_filter, &filt);
  const int lcap = need <= 64 ? 64 : need <= 256 ? 256 : need <= 1024 ? 1024 : 0;
  if (!lcap) return fail(DG_ENOTSUP, "beam width / expanded beam above 1024 is not supported");
  if (reranked && !filt && search_k > 1024) return fail(DG_ENOTSUP, "rerank size above 1024");
  const uint32_t hbits = visited_bits(idx, trav, lcap, filt, maxL);
  uint32_t hB = 1;
  while (hB < 32 && (1ull << hB) < idx->n) ++hB;
  hB = std::max(hB, hbits);

  // scratch layout: [0, 256) work counter | filter ops | offsets | pool | beams | per-query k
  auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const size_t o_ops = 256;
  const size_t o_offs = o_ops + up16(any_filter ? (size_t)total_ops * sizeof(DgFilterOp) : 0);
  const size_t o_pool = o_offs + up16(any_filter && p->filter_offsets ? (size_t)(nq + 1) * 4 : 0);
  const size_t o_beam = o_pool + up16(any_filter ? (size_t)p->filter_pool_len * 8 : 0);
  const size_t o_k = o_beam + up16(p->per_query_beam ? (size_t)nq * 4 : 0);
  const size_t used = o_k + up16(p->per_query_k ? (size_t)nq * 4 : 0);
  if (used > kStaticScratchBytes)
    return fail(DG_EINVAL, "per-call parameters need " + std::to_string(used) + " bytes; the static scratch holds " +
                               std::to_string(kStaticScratchBytes) + " (fewer filter ops or per-query beams per call)");

  std::lock_guard<std::mutex> lk(idx->mu);
  DG_CUDA(cudaSetDevice(idx->device));
  unsigned char *scratch = nullptr;
  DgStatus s = static_scratch(idx->device, &scratch);
  if (s != DG_OK) return s;
  cudaStream_t st = (p->flags & DG_FLAG_STREAM) || p->stream ? (cudaStream_t)p->stream : idx->stream;

  SearchArgs a{};
  a.n = idx->n;
  a.d = idx->d;
  a.dpad = idx->dpad;
  a.R = idx->R;
  a.medoid = idx->medoid;
  index_state(idx, a);
  a.metric = idx->metric;
  a.vec_f32 = idx->vec;
  a.vec_bf16 = idx->bf16;
  a.bf16_n2 = idx->bf16_n2;
  a.adj = idx->adj;
  a.codes = idx->codes;
  a.code_stride = idx->code_stride;
  a.pq_M = idx->pq_M;
  a.pq_K = idx->pq_K;
  a.pq_ds = idx->pq_M ? idx->d / idx->pq_M : 0;
  a.pq_cb = idx->pq_cb;
  a.i8_scale = idx->i8_scale;
  a.i8_offset = idx->i8_offset;
  a.i8_norm = idx->i8_norm;
  a.i8_sum = idx->i8_sum;
  a.vec_fp8 = idx->fp8;
  a.fp8_sn = idx->fp8_sn;
  a.rq_padded = idx->rq_padded;
  a.rq_centroid = idx->rq_centroid;
  a.rq_signs = idx->rq_signs;
  a.dnorm2 = idx->dnorm2;
  a.labels = idx->labels;
  a.nf = idx->nf;
  a.nq = nq;
  a.k = p->k;
  a.L = p->beam_width;
  a.rerank = p->rerank_size;
  a.hbits = hbits;
  a.hB = hB;
  // every call reuses the array: the counter must start at zero again
  DG_CUDA(cudaMemsetAsync(scratch, 0, 4, st));
  a.counter = reinterpret_cast<uint32_t *>(scratch);
  if (any_filter) {
    DG_CUDA(cudaMemcpyAsync(scratch + o_ops, p->filter_ops, (size_t)total_ops * sizeof(DgFilterOp),
                            cudaMemcpyHostToDevice, st));
    a.fops = reinterpret_cast<const DgFilterOp *>(scratch + o_ops);
    a.fnops = p->filter_offsets ? 0 : p->filter_nops;
    if (p->filter_offsets) {
      DG_CUDA(cudaMemcpyAsync(scratch + o_offs, p->filter_offsets, (size_t)(nq + 1) * 4, cudaMemcpyHostToDevice, st));
      a.foffs = reinterpret_cast<const uint32_t *>(scratch + o_offs);
    }
    if (p->filter_pool_len)
      DG_CUDA(cudaMemcpyAsync(scratch + o_pool, p->filter_pool, (size_t)p->filter_pool_len * 8,
                              cudaMemcpyHostToDevice, st));
    a.fpool = reinterpret_cast<const uint64_t *>(scratch + o_pool);
  }
  if (p->per_query_beam) {
    DG_CUDA(cudaMemcpyAsync(scratch + o_beam, p->per_query_beam, (size_t)nq * 4, cudaMemcpyHostToDevice, st));
    a.perL = reinterpret_cast<const uint32_t *>(scratch + o_beam);
  }
  if (p->per_query_k) {
    DG_CUDA(cudaMemcpyAsync(scratch + o_k, p->per_query_k, (size_t)nq * 4, cudaMemcpyHostToDevice, st));
    a.perK = reinterpret_cast<const uint32_t *>(scratch + o_k);
  }
  a.Q = queries;
  a.out_ids = out_ids;
  a.out_d = out_dists;
  a.out_cnt = out_counts;
  a.out_stats = nullptr;

  const int met = met_kind(idx->metric);
  int lpr = 1;
  if (trav == TRAV_F32) lpr = 8;
  else if (trav == TRAV_BF16 || trav == TRAV_F16) lpr = lanes_per_row(idx->dpad / 8);
  else if (trav == TRAV_INT8) lpr = lanes_per_row(idx->code_stride / 16);
  const WarpLayout Ly = warp_layout(trav, lcap, filt, hbits, idx->dpad, idx->pq_M, idx->pq_K,
                                    idx->rq_padded,
                                    (trav == TRAV_RABITQ || trav == TRAV_INT8) && met_kind(idx->metric) != MET_L2,
                                    idx->R, true);
  LaunchInfo info;
  switch (trav) {
    case TRAV_F32: s = launch_search_f32(a, Ly, met, lpr, lcap, filt, st, &info); break;
    case TRAV_BF16: s = launch_search_bf16(a, Ly, met, lpr, lcap, filt, st, &info); break;
    case TRAV_F16: s = launch_search_f16(a, Ly, met, lpr, lcap, filt, st, &info); break;
    case TRAV_INT8: s = launch_search_int8(a, Ly, met, lpr, lcap, filt, st, &info); break;
    case TRAV_PQ: s = launch_search_pq(a, Ly, met, lpr, lcap, filt, st, &info); break;
    case TRAV_FP8: s = launch_search_fp8(a, Ly, met, lpr, lcap, filt, st, &info); break;
    default: s = launch_search_rabitq(a, Ly, met, lpr, lcap, filt, st, &info); break;
  }
  if (s != DG_OK) return s;
  // Record the search's completion on a slot event (created with the index,
  // so nothing is allocated here): updates of rows, adjacency, labels or
  // tombstones and dg_index_destroy wait for it, as they do for dg_search_batch.
  DgIndex::Slot *slp = nullptr;
  DG_CUDA(take_slot(idx, &slp));
  DG_CUDA(cudaEventRecord(slp->done, st));
  slp->pending = true;
  return DG_OK;
}
