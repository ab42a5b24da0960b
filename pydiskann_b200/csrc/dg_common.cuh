// dg_common.cuh -- shared device utilities of libdgann (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <stdint.h>

#include <string>

#include "../../include/dgann.h"

namespace dg {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint64_t kKeyInvalid = ~0ull;

// Host-side error state (thread local) and CUDA error mapping.
void set_error(const std::string &msg);
DgStatus fail(DgStatus st, const std::string &msg);
DgStatus cuda_fail(cudaError_t e, const char *what);

#define DG_CUDA(call)                                      \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return ::dg::cuda_fail(e_, #call); \
  } while (0)

// ------------------------------------------------------------------ keys
// A candidate is one 64-bit key: order-preserving distance bits in the high
// word, node id in bits 1..31 and the "expanded" flag in bit 0.  Unsigned key
// order is therefore (distance, id) lexicographic, the tie rule shared with
// the oracle, and the flag never changes the order of two distinct nodes.
__device__ __forceinline__ uint32_t ordered_bits(float d) {
  if (d == 0.0f) d = 0.0f;  // -0 -> +0
  uint32_t u = __float_as_uint(d);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_dist(uint64_t key) {
  uint32_t u = (uint32_t)(key >> 32);
  u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  return __uint_as_float(u);
}
__device__ __forceinline__ uint32_t key_hi(uint64_t key) { return (uint32_t)(key >> 32); }
__device__ __forceinline__ uint32_t key_id(uint64_t key) { return ((uint32_t)key) >> 1; }
__device__ __forceinline__ bool key_expanded(uint64_t key) { return key & 1ull; }
__device__ __forceinline__ uint64_t make_key(float d, uint32_t id) {
  return ((uint64_t)ordered_bits(d) << 32) | ((uint64_t)id << 1);
}
// Key with an explicit 31-bit payload (used for rank-ordered rerank lists).
__device__ __forceinline__ uint64_t make_key_payload(float d, uint32_t payload) {
  return ((uint64_t)ordered_bits(d) << 32) | ((uint64_t)payload << 1);
}
__device__ __forceinline__ uint64_t strip_flag(uint64_t key) { return key & ~1ull; }

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
  uint32_t lo = __shfl_sync(kFull, (uint32_t)v, src);
  uint32_t hi = __shfl_sync(kFull, (uint32_t)(v >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
  uint32_t lo = __shfl_xor_sync(kFull, (uint32_t)v, m);
  uint32_t hi = __shfl_xor_sync(kFull, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}

// Ascending bitonic sort of one key per lane across the warp.
__device__ __forceinline__ uint64_t warp_sort_keys(uint64_t key, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      uint64_t other = shfl_xor64(key, j);
      bool up = ((lane & k) == 0);
      bool lower = ((lane & j) == 0);
      // lower lane keeps min when ascending block, max when descending block
      bool take_min = (lower == up);
      uint64_t mn = other < key ? other : key;
      uint64_t mx = other < key ? key : other;
      key = take_min ? mn : mx;
    }
  }
  return key;
}

// Sum across the LPR lanes of each lane group, transposed: p[i] on entry is
// this lane's partial for item i (i < LPR); on exit lane r of a group holds
// the group total of item r.
template <int LPR, typename T>
__device__ __forceinline__ T transpose_reduce(T (&p)[LPR], int lane) {
#pragma unroll
  for (int s = LPR / 2; s >= 1; s >>= 1) {
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int i = 0; i < s; ++i) {
      T send = upper ? p[i] : p[i + s];
      T keep = upper ? p[i + s] : p[i];
      p[i] = keep + __shfl_xor_sync(kFull, send, s);
    }
  }
  return p[0];
}

// ------------------------------------------------------- counter-based RNG
// splitmix64 finaliser chained over (seed, a, b, c); the oracle uses the same
// stream so a GPU build and an oracle build draw identical numbers.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t rand4(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
  return mix64(mix64(mix64(seed + a) + b) + c);
}
__device__ __forceinline__ uint64_t range_of(uint64_t r, uint64_t n) { return __umul64hi(r, n); }

// ------------------------------------------------------------------ filter
// Postfix evaluation of a DgFilterOp program over one label row
// (Filter::matches, src/filtered.rs:120-135).
constexpr int kFilterStack = 32;
__device__ __forceinline__ bool filter_eval(const DgFilterOp *prog, uint32_t nops,
                                            const uint64_t *pool, const uint64_t *labels,
                                            uint32_t nf) {
  if (nops == 0) return true;
  uint32_t stack = 0;  // bit stack
  int sp = 0;
  for (uint32_t i = 0; i < nops; ++i) {
    const DgFilterOp o = prog[i];
    bool v = false;
    switch (o.op) {
      case DG_F_TRUE: v = true; break;
      case DG_F_EQ: v = o.field < nf && labels[o.field] == o.a; break;
      case DG_F_IN:
        if (o.field < nf) {
          const uint64_t x = labels[o.field];
          for (uint64_t t = 0; t < o.b; ++t)
            if (pool[o.a + t] == x) { v = true; break; }
        }
        break;
      case DG_F_LT: v = o.field < nf && labels[o.field] < o.a; break;
      case DG_F_GT: v = o.field < nf && labels[o.field] > o.a; break;
      case DG_F_RANGE: v = o.field < nf && labels[o.field] >= o.a && labels[o.field] <= o.b; break;
      case DG_F_AND:
      case DG_F_OR: {
        bool acc = o.op == DG_F_AND;
        for (uint32_t t = 0; t < o.field && sp > 0; ++t) {
          --sp;
          bool x = (stack >> sp) & 1u;
          acc = (o.op == DG_F_AND) ? (acc && x) : (acc || x);
        }
        v = acc;
        break;
      }
      default: v = false;
    }
    if (sp < kFilterStack) {
      stack = v ? (stack | (1u << sp)) : (stack & ~(1u << sp));
      ++sp;
    }
  }
  return sp > 0 ? ((stack >> (sp - 1)) & 1u) : true;
}

}  // namespace dg
