// dg_serve.cu -- continuous-batching request loop over a DgIndex.
//
// Requests (one query each, with its own k, beam, rerank, traversal and
// filter) are queued by dg_server_submit.  A dispatcher thread forms batches
// of pending requests that share (traversal, rerank, filter presence) -- k,
// beam and the filter program stay per request, so one launch carries uneven
// k, beams and filters -- and launches each batch on the next free stream
// slot; a request that arrives while other batches are on the GPU goes into
// the next batch as soon as a slot and memory are free, and batches on
// different slots run concurrently on the device.
//
// Admission by HBM budget: the server holds one device arena (and a pinned
// host arena of the same size) of hbm_budget_bytes, allocated at creation.
// Each batch takes a region sized by its own need -- its queries, its result
// rows at the batch's largest k, its per-query beams and k -- first fit; a
// batch that does not fit is trimmed to the requests that do, and when not
// even one fits the dispatcher waits for batches in flight to return their
// regions.  A host function enqueued after each batch's result copy completes
// its requests and frees its region; dg_server_wait waits for a ticket with a
// bound.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dg_index.h"

namespace dg {

using Clock = std::chrono::steady_clock;

struct ServeRequest {
  uint64_t ticket = 0;  // (generation << 32) | slot
  uint32_t slot = 0, gen = 1;
  bool live = false;    // submitted and not yet waited for
  std::vector<float> query;
  uint32_t k = 10, beam = 64, rerank = 0;
  int32_t traversal = DG_TRAVERSE_F32;
  std::vector<DgFilterOp> ops;
  std::vector<uint64_t> pool;
  Clock::time_point arrival, done_at;
  bool done = false;
  bool picked = false;  // taken into the batch being formed (under the server's mutex)
  DgStatus status = DG_OK;
  std::string err;  // dg_last_error of the dispatcher thread when status != DG_OK
  std::vector<uint32_t> ids;
  std::vector<float> dists;
  uint32_t count = 0;
};

// A batch's region of the arenas (offsets into the device and pinned host
// arenas; the same layout in both):
//   queries f32[nq*d] | ids u32[nq*k] dists f32[nq*k] counts u32[nq] | beams u32[nq] | k u32[nq]
// with k the batch's largest; every part starts on 256 bytes.
struct BatchLayout {
  size_t q = 0, out = 0, beam = 0, kq = 0, bytes = 0;
};
inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
inline BatchLayout batch_layout(uint32_t nq, uint32_t d, uint32_t kmax) {
  BatchLayout L;
  L.q = 0;
  L.out = up256((size_t)nq * d * 4);
  L.beam = L.out + up256((size_t)nq * kmax * 8 + (size_t)nq * 4);
  L.kq = L.beam + up256((size_t)nq * 4);
  L.bytes = L.kq + up256((size_t)nq * 4);
  return L;
}

// First-fit allocator over [0, cap) (under the server's mutex).
struct Arena {
  size_t cap = 0;
  std::vector<std::pair<size_t, size_t>> used;  // (offset, bytes), sorted by offset
  bool take(size_t bytes, size_t *off) {
    size_t at = 0;
    for (size_t i = 0; i <= used.size(); ++i) {
      const size_t end = i < used.size() ? used[i].first : cap;
      if (end >= at && end - at >= bytes) {
        used.insert(used.begin() + i, {at, bytes});
        *off = at;
        return true;
      }
      if (i < used.size()) at = used[i].first + used[i].second;
    }
    return false;
  }
  void give(size_t off) {
    for (size_t i = 0; i < used.size(); ++i)
      if (used[i].first == off) {
        used.erase(used.begin() + i);
        return;
      }
  }
  size_t in_use() const {
    size_t t = 0;
    for (auto &u : used) t += u.second;
    return t;
  }
};

struct ServeSlot {
  cudaStream_t stream = nullptr;
  bool busy = false;
  std::vector<ServeRequest *> batch;
  uint32_t k = 0;       // result row stride: the batch's largest k
  size_t off = 0;       // the batch's arena region
  // pinned staging of the batch's filter programs (ops, offsets, IN pool),
  // sized at creation: a copy from pageable memory is staged by the driver
  // through a shared buffer and can wait behind other streams' kernels
  DgFilterOp *h_ops = nullptr;
  uint32_t *h_offs = nullptr;
  uint64_t *h_pool = nullptr;
  size_t cap_ops = 0, cap_pool = 0;
};

}  // namespace dg

struct DgServer {
  DgIndex *idx = nullptr;
  DgServerConfig cfg{};
  std::vector<dg::ServeSlot> slots;
  dg::Arena arena;                          // under mu
  uint8_t *d_arena = nullptr, *h_arena = nullptr;
  size_t peak_bytes = 0;                    // largest arena use seen (under mu)
  std::mutex mu;
  std::condition_variable cv_submit, cv_done, cv_slot;
  std::deque<dg::ServeRequest *> pending;
  bool stop = false;
  std::thread dispatcher;
  std::atomic<uint64_t> batches{0}, served{0};
  uint32_t in_flight = 0, max_in_flight = 0;  // busy slots (under mu)
  DgStatus fatal = DG_OK;
  std::string fatal_msg;
  // Request records, reused (with their buffers) by later requests so that no
  // allocation happens per request once the server has warmed up; a ticket
  // names a record slot and its generation.
  std::mutex pool_mu;
  std::vector<dg::ServeRequest *> recs;
  std::vector<uint32_t> free_slots;
};

namespace dg {

static ServeRequest *take_request(DgServer *s) {
  std::lock_guard<std::mutex> lk(s->pool_mu);
  if (!s->free_slots.empty()) {
    ServeRequest *r = s->recs[s->free_slots.back()];
    s->free_slots.pop_back();
    return r;
  }
  ServeRequest *r = new (std::nothrow) ServeRequest();
  if (!r) return nullptr;
  r->slot = (uint32_t)s->recs.size();
  s->recs.push_back(r);
  return r;
}

static ServeRequest *record_of(DgServer *s, uint64_t ticket) {
  const uint32_t slot = (uint32_t)ticket;
  std::lock_guard<std::mutex> lk(s->pool_mu);
  return slot < s->recs.size() ? s->recs[slot] : nullptr;
}

static void give_request(DgServer *s, ServeRequest *r) {
  r->done = false;
  r->status = DG_OK;
  r->err.clear();
  r->ops.clear();
  r->pool.clear();
  r->count = 0;
  r->live = false;
  ++r->gen;
  std::lock_guard<std::mutex> lk(s->pool_mu);
  s->free_slots.push_back(r->slot);
}

struct SlotDone {
  DgServer *s;
  int slot;
};

// Runs on the driver's callback thread once the slot's result copies landed;
// it only touches host memory.
static void CUDART_CB slot_done(void *arg) {
  SlotDone *sd = static_cast<SlotDone *>(arg);
  DgServer *s = sd->s;
  ServeSlot &sl = s->slots[sd->slot];
  const auto now = Clock::now();
  // results into the requests' own buffers (sized at submission) without the
  // lock: a waiter reads them only after seeing `done`, which is set below
  const size_t nb = sl.batch.size(), nk = nb * (size_t)sl.k;
  const BatchLayout L = batch_layout((uint32_t)nb, s->idx->d, sl.k);
  const uint8_t *h_out = s->h_arena + sl.off + L.out;
  const uint32_t *ids = reinterpret_cast<const uint32_t *>(h_out);
  const float *ds = reinterpret_cast<const float *>(h_out + nk * 4);
  const uint32_t *cnt = reinterpret_cast<const uint32_t *>(h_out + nk * 8);
  for (size_t i = 0; i < nb; ++i) {
    ServeRequest *r = sl.batch[i];
    r->count = std::min(cnt[i], r->k);
    std::memcpy(r->ids.data(), ids + i * sl.k, r->k * sizeof(uint32_t));
    std::memcpy(r->dists.data(), ds + i * sl.k, r->k * sizeof(float));
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (ServeRequest *r : sl.batch) {
      r->done_at = now;
      r->done = true;
    }
    s->served += nb;
    sl.batch.clear();
    sl.busy = false;
    s->arena.give(sl.off);
    --s->in_flight;
  }
  s->cv_done.notify_all();
  s->cv_slot.notify_all();
  delete sd;
}

static bool same_class(const ServeRequest *a, const ServeRequest *b) {
  // a filtered search is a different traversal (expanded beam), so requests
  // with and without a filter never share a batch; k, beam and the filter
  // program are per query within a launch
  return a->traversal == b->traversal && a->rerank == b->rerank && a->ops.empty() == b->ops.empty();
}

// Fails one request (under mu).
static void fail_request(DgServer *s, ServeRequest *r, DgStatus st, const std::string &why) {
  r->status = st;
  r->err = why;
  r->done = true;
  r->done_at = Clock::now();
  s->cv_done.notify_all();
}

static void dispatch_loop(DgServer *s) {
  const uint32_t dim = s->idx->d;
  std::vector<uint32_t> offs;
  std::vector<ServeRequest *> batch;
  std::vector<DgFilterOp> ops;
  std::vector<uint64_t> pool;
  cudaSetDevice(s->idx->device);
  while (true) {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_submit.wait(lk, [&] { return s->stop || !s->pending.empty(); });
    if (s->stop && s->pending.empty()) break;
    // give a partial batch a short time to fill
    if (s->pending.size() < s->cfg.max_batch && s->cfg.max_wait_us > 0) {
      const auto deadline = s->pending.front()->arrival + std::chrono::microseconds(s->cfg.max_wait_us);
      s->cv_submit.wait_until(lk, deadline, [&] { return s->stop || s->pending.size() >= s->cfg.max_batch; });
    }
    // a free slot (a stream for the batch)
    int slot = -1;
    s->cv_slot.wait(lk, [&] {
      for (size_t i = 0; i < s->slots.size(); ++i)
        if (!s->slots[i].busy) {
          slot = (int)i;
          return true;
        }
      return s->stop;
    });
    if (slot < 0) break;
    ServeSlot &sl = s->slots[slot];
    // oldest request fixes the class; candidates: up to max_batch of that
    // class in arrival order
    ServeRequest *head = s->pending.front();
    batch.clear();
    for (auto it = s->pending.begin(); it != s->pending.end() && batch.size() < s->cfg.max_batch; ++it)
      if (same_class(*it, head)) batch.push_back(*it);
    // admission: the longest prefix of the candidates whose region fits
    size_t off = 0;
    uint32_t take = (uint32_t)batch.size(), kmax = 0;
    while (take > 0) {
      kmax = 0;
      for (uint32_t i = 0; i < take; ++i) kmax = std::max(kmax, batch[i]->k);
      if (s->arena.take(batch_layout(take, dim, kmax).bytes, &off)) break;
      take = take > 8 ? take - take / 4 : take - 1;
    }
    if (take == 0) {
      if (s->in_flight == 0) {  // cannot fit even alone: the budget is too small for it
        ServeRequest *r = head;
        s->pending.erase(std::find(s->pending.begin(), s->pending.end(), r));
        fail_request(s, r, DG_ENOMEM, "request needs more memory than the server's HBM budget");
        continue;
      }
      // wait for a batch in flight to return its region
      const uint64_t served0 = s->served.load();
      s->cv_slot.wait(lk, [&] { return s->stop || s->served.load() != served0 || s->in_flight == 0; });
      continue;
    }
    batch.resize(take);
    for (ServeRequest *r : batch) r->picked = true;
    s->pending.erase(std::remove_if(s->pending.begin(), s->pending.end(), [](ServeRequest *r) { return r->picked; }),
                     s->pending.end());
    for (ServeRequest *r : batch) r->picked = false;
    sl.busy = true;
    sl.off = off;
    s->peak_bytes = std::max(s->peak_bytes, s->arena.in_use());
    s->max_in_flight = std::max(s->max_in_flight, ++s->in_flight);
    sl.batch = batch;
    sl.k = kmax;
    lk.unlock();

    const uint32_t nq = (uint32_t)batch.size();
    const BatchLayout L = batch_layout(nq, dim, kmax);
    float *h_q = reinterpret_cast<float *>(s->h_arena + off + L.q);
    uint32_t *h_beam = reinterpret_cast<uint32_t *>(s->h_arena + off + L.beam);
    uint32_t *h_k = reinterpret_cast<uint32_t *>(s->h_arena + off + L.kq);
    float *d_q = reinterpret_cast<float *>(s->d_arena + off + L.q);
    uint8_t *d_out = s->d_arena + off + L.out;
    offs.assign(1, 0);
    ops.clear();
    pool.clear();
    bool any_filter = false;
    for (uint32_t i = 0; i < nq; ++i) {
      ServeRequest *r = batch[i];
      std::memcpy(h_q + (size_t)i * dim, r->query.data(), dim * sizeof(float));
      h_beam[i] = r->beam;
      h_k[i] = r->k;
      const uint64_t base = pool.size();
      for (DgFilterOp o : r->ops) {
        if (o.op == DG_F_IN) o.a += base;
        ops.push_back(o);
      }
      pool.insert(pool.end(), r->pool.begin(), r->pool.end());
      any_filter |= !r->ops.empty();
      offs.push_back((uint32_t)ops.size());
    }
    DgStatus st = DG_OK;
    if (cudaMemcpyAsync(d_q, h_q, (size_t)nq * dim * sizeof(float), cudaMemcpyHostToDevice, sl.stream) !=
        cudaSuccess)
      st = fail(DG_EDEVICE, "request copy failed");
    if (st == DG_OK) {
      DgSearchParams p{};
      p.k = kmax;
      p.beam_width = head->beam;
      p.rerank_size = head->rerank;
      p.traversal = head->traversal;
      p.per_query_beam = h_beam;
      p.per_query_k = h_k;
      if (any_filter) {
        p.filter_ops = ops.data();
        p.filter_offsets = offs.data();
        p.filter_pool = pool.data();
        p.filter_pool_len = (uint32_t)pool.size();
        if (ops.size() <= sl.cap_ops && pool.size() <= sl.cap_pool && sl.h_ops) {
          std::memcpy(sl.h_ops, ops.data(), ops.size() * sizeof(DgFilterOp));
          std::memcpy(sl.h_offs, offs.data(), offs.size() * sizeof(uint32_t));
          if (!pool.empty()) std::memcpy(sl.h_pool, pool.data(), pool.size() * sizeof(uint64_t));
          p.filter_ops = sl.h_ops;
          p.filter_offsets = sl.h_offs;
          p.filter_pool = sl.h_pool;
        }
      }
      p.flags = DG_FLAG_DEVICE_PTRS | DG_FLAG_STREAM;
      p.stream = sl.stream;
      const size_t nk = (size_t)nq * kmax;
      st = dg_search_batch(s->idx, &p, d_q, nq, reinterpret_cast<uint32_t *>(d_out),
                           reinterpret_cast<float *>(d_out + nk * 4), reinterpret_cast<uint32_t *>(d_out + nk * 8),
                           nullptr);
    }
    if (st == DG_OK) {
      const size_t kq = (size_t)nq * kmax;
      if (cudaMemcpyAsync(s->h_arena + off + L.out, d_out, kq * 8 + (size_t)nq * 4, cudaMemcpyDeviceToHost,
                          sl.stream) != cudaSuccess ||
          cudaLaunchHostFunc(sl.stream, slot_done, new SlotDone{s, slot}) != cudaSuccess)
        st = fail(DG_EDEVICE, "result copy failed");
    }
    ++s->batches;
    if (st != DG_OK) {  // fail the batch's requests, free the slot
      const std::string why = dg_last_error();
      std::lock_guard<std::mutex> g(s->mu);
      for (ServeRequest *r : batch) {
        r->status = st;
        r->err = why;
        r->done = true;
        r->done_at = Clock::now();
      }
      sl.batch.clear();
      sl.busy = false;
      cudaStreamSynchronize(sl.stream);  // the region may be read by copies already issued
      s->arena.give(off);
      --s->in_flight;
      s->cv_done.notify_all();
      s->cv_slot.notify_all();
    }
  }
}

static DgStatus check_request(const DgServer *s, const float *query, const DgRequest *rq) {
  if (!query || !rq) return fail(DG_EINVAL, "null request");
  if (rq->k == 0 || rq->k > s->cfg.max_k) return fail(DG_EINVAL, "k must be in [1, max_k]");
  if (rq->beam_width == 0) return fail(DG_EINVAL, "beam_width must be >= 1");
  if (rq->filter_nops > s->cfg.max_filter_ops) return fail(DG_EINVAL, "filter program above max_filter_ops");
  if (rq->filter_nops && !rq->filter_ops) return fail(DG_EINVAL, "filter ops missing");
  if (rq->filter_pool_len && !rq->filter_pool) return fail(DG_EINVAL, "filter pool missing");
  return DG_OK;
}

static DgStatus copy_request(const DgServer *s, const float *query, const DgRequest *rq, ServeRequest *r) {
  const DgStatus st = check_request(s, query, rq);
  if (st != DG_OK) return st;
  r->query.assign(query, query + s->idx->d);
  r->k = rq->k;
  r->ids.resize(rq->k);
  r->dists.resize(rq->k);
  r->beam = rq->beam_width;
  r->rerank = rq->rerank_size;
  r->traversal = rq->traversal;
  if (rq->filter_nops) {
    r->ops.assign(rq->filter_ops, rq->filter_ops + rq->filter_nops);
    if (rq->filter_pool_len) r->pool.assign(rq->filter_pool, rq->filter_pool + rq->filter_pool_len);
  }
  return DG_OK;
}

}  // namespace dg

using namespace dg;

extern "C" {

DgStatus dg_server_destroy(DgServer *s) {
  if (!s) return DG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_submit.notify_all();
  s->cv_slot.notify_all();
  if (s->dispatcher.joinable()) s->dispatcher.join();
  cudaSetDevice(s->idx->device);
  for (ServeSlot &sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    for (void *h : {(void *)sl.h_ops, (void *)sl.h_offs, (void *)sl.h_pool})
      if (h) cudaFreeHost(h);
  }
  if (s->h_arena) cudaFreeHost(s->h_arena);
  if (s->d_arena) cudaFree(s->d_arena);
  for (ServeRequest *r : s->recs) delete r;
  delete s;
  return DG_OK;
}

DgStatus dg_server_create(DgIndex *idx, const DgServerConfig *cfg, DgServer **out) {
  if (!idx || !cfg || !out) return fail(DG_EINVAL, "null argument");
  *out = nullptr;
  if (cfg->max_batch == 0 || cfg->streams == 0 || cfg->max_k == 0)
    return fail(DG_EINVAL, "max_batch, streams and max_k must be >= 1");
  // arena: the budget, or (without one) room for a full batch at max_k on every stream
  const size_t full = batch_layout(cfg->max_batch, idx->d, cfg->max_k).bytes;
  const size_t one = batch_layout(1, idx->d, cfg->max_k).bytes;
  const size_t arena = cfg->hbm_budget_bytes ? (size_t)cfg->hbm_budget_bytes : full * cfg->streams;
  if (arena < one)
    return fail(DG_ENOMEM, "HBM budget (" + std::to_string(arena) + " bytes) below one request at max_k (" +
                               std::to_string(one) + " bytes)");
  DG_CUDA(cudaSetDevice(idx->device));
  DgServer *s = new (std::nothrow) DgServer();
  if (!s) return fail(DG_ENOMEM, "host allocation failed");
  s->idx = idx;
  s->cfg = *cfg;
  s->arena.cap = arena;
  if (cudaMalloc(&s->d_arena, arena) != cudaSuccess || cudaMallocHost(&s->h_arena, arena) != cudaSuccess) {
    dg_server_destroy(s);
    return fail(DG_ENOMEM, "server arena allocation failed");
  }
  // the index's per-call staging at this server's largest batch, so no batch
  // reallocates it (and synchronises the device) while others are in flight
  DgStatus rs = reserve_call_buffers(idx, cfg->max_batch, (size_t)cfg->max_batch * cfg->max_filter_ops,
                                     (size_t)cfg->max_batch * cfg->max_filter_ops);
  if (rs != DG_OK) {
    dg_server_destroy(s);
    return rs;
  }
  s->slots.resize(cfg->streams);
  for (ServeSlot &sl : s->slots) {
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess) {
      dg_server_destroy(s);
      return fail(DG_EDEVICE, "server stream creation failed");
    }
    if (cfg->max_filter_ops) {
      sl.cap_ops = sl.cap_pool = (size_t)cfg->max_batch * cfg->max_filter_ops;
      if (cudaMallocHost((void **)&sl.h_ops, sl.cap_ops * sizeof(DgFilterOp)) != cudaSuccess ||
          cudaMallocHost((void **)&sl.h_offs, ((size_t)cfg->max_batch + 1) * sizeof(uint32_t)) != cudaSuccess ||
          cudaMallocHost((void **)&sl.h_pool, sl.cap_pool * sizeof(uint64_t)) != cudaSuccess) {
        dg_server_destroy(s);
        return fail(DG_ENOMEM, "server filter staging allocation failed");
      }
    }
  }
  s->dispatcher = std::thread(dispatch_loop, s);
  *out = s;
  return DG_OK;
}

DgStatus dg_server_submit(DgServer *s, const float *query, const DgRequest *req, uint64_t *ticket) {
  if (!s || !ticket) return fail(DG_EINVAL, "null argument");
  ServeRequest *r = take_request(s);
  if (!r) return fail(DG_ENOMEM, "host allocation failed");
  DgStatus st = copy_request(s, query, req, r);
  if (st != DG_OK) {
    give_request(s, r);
    return st;
  }
  r->arrival = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;  // not returned to the pool: the server is going away
      return fail(DG_EINVAL, "server is shutting down");
    }
    r->ticket = ((uint64_t)r->gen << 32) | r->slot;
    r->live = true;
    s->pending.push_back(r);
    *ticket = r->ticket;
  }
  s->cv_submit.notify_one();
  return DG_OK;
}

DgStatus dg_server_wait(DgServer *s, uint64_t ticket, int64_t timeout_us, uint32_t *out_ids, float *out_dists,
                        uint32_t *out_count, double *latency_us) {
  if (!s) return fail(DG_EINVAL, "null server");
  ServeRequest *r = record_of(s, ticket);
  std::unique_lock<std::mutex> lk(s->mu);
  if (!r || !r->live || r->ticket != ticket) return fail(DG_EINVAL, "unknown ticket");
  const auto deadline = Clock::now() + std::chrono::microseconds(timeout_us < 0 ? 0 : timeout_us);
  if (!s->cv_done.wait_until(lk, deadline, [&] { return r->done; }))
    return fail(DG_ETIMEOUT, "request " + std::to_string(ticket) + " not done within the wait bound");
  r->live = false;
  lk.unlock();
  const DgStatus st = r->status;
  if (st != DG_OK) fail(st, r->err);
  if (st == DG_OK) {
    if (out_ids) std::copy(r->ids.begin(), r->ids.end(), out_ids);
    if (out_dists) std::copy(r->dists.begin(), r->dists.end(), out_dists);
    if (out_count) *out_count = r->count;
    if (latency_us)
      *latency_us = std::chrono::duration<double, std::micro>(r->done_at - r->arrival).count();
  }
  give_request(s, r);
  return st;
}

DgStatus dg_server_stats(DgServer *s, uint64_t *batches, uint64_t *served, uint32_t *max_in_flight) {
  if (!s) return fail(DG_EINVAL, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (batches) *batches = s->batches.load();
  if (served) *served = s->served.load();
  if (max_in_flight) *max_in_flight = s->max_in_flight;
  return DG_OK;
}

// Replays an arrival trace from a native thread: request i is submitted at
// arrival_us[i] (relative to the start) and its latency is written to
// latency_us[i]; results to out_ids/out_dists (k-strided per request) and
// out_counts.  Returns once every request completed or timeout_us passed.
DgStatus dg_server_run_trace(DgServer *s, const float *queries, uint32_t n, const DgRequest *reqs,
                             const double *arrival_us, int64_t timeout_us, uint32_t *out_ids, float *out_dists,
                             uint32_t *out_counts, double *latency_us, double *wall_us) {
  if (!s || !queries || !reqs || !arrival_us || !latency_us) return fail(DG_EINVAL, "null argument");
  for (uint32_t i = 0; i < n; ++i) {
    const DgStatus st = check_request(s, queries + (size_t)i * s->idx->d, &reqs[i]);
    if (st != DG_OK) return fail(st, "request " + std::to_string(i) + ": " + dg_last_error());
  }
  std::vector<uint64_t> tickets(n, 0);
  std::atomic<int> submit_err{0};
  const auto t0 = Clock::now();
  auto sched = [&](uint32_t i) {
    return t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::micro>(arrival_us[i]));
  };
  // Every request that is due is queued in one critical section; its arrival
  // is its scheduled time, so latency counts any submission delay.
  std::thread producer([&] {
    std::vector<ServeRequest *> due;
    uint32_t i = 0;
    while (i < n) {
      const auto at = sched(i);
      while (Clock::now() < at) {
        const auto left = at - Clock::now();
        if (left > std::chrono::microseconds(50)) std::this_thread::sleep_for(left - std::chrono::microseconds(30));
      }
      const auto now = Clock::now();
      const uint32_t i0 = i;
      due.clear();
      while (i < n && sched(i) <= now && due.size() < 1024) {
        ServeRequest *r = take_request(s);
        if (!r || copy_request(s, queries + (size_t)i * s->idx->d, &reqs[i], r) != DG_OK) {
          if (r) give_request(s, r);
          for (ServeRequest *x : due) give_request(s, x);
          submit_err = 1;
          return;
        }
        r->arrival = sched(i);
        due.push_back(r);
        ++i;
      }
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
          for (ServeRequest *r : due) give_request(s, r);
          submit_err = 1;
          return;
        }
        for (size_t j = 0; j < due.size(); ++j) {
          ServeRequest *r = due[j];
          r->ticket = ((uint64_t)r->gen << 32) | r->slot;
          r->live = true;
          s->pending.push_back(r);
          tickets[i0 + j] = r->ticket;
        }
      }
      s->cv_submit.notify_one();
    }
  });
  producer.join();
  if (submit_err) return fail(DG_EINVAL, "the server stopped while the trace was submitted");
  DgStatus st = DG_OK;
  size_t off = 0;
  double last_done = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    const int64_t left = timeout_us - (int64_t)std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    DgStatus r = dg_server_wait(s, tickets[i], std::max<int64_t>(left, 0), out_ids ? out_ids + off : nullptr,
                                out_dists ? out_dists + off : nullptr, out_counts ? out_counts + i : nullptr,
                                latency_us + i);
    off += reqs[i].k;
    if (r != DG_OK) latency_us[i] = -1.0;
    if (r != DG_OK && st == DG_OK) st = r;
    if (r == DG_OK) last_done = std::max(last_done, arrival_us[i] + latency_us[i]);
  }
  if (wall_us) *wall_us = last_done;
  return st;
}

}  // extern "C"
