// dg_build.cu -- encoders, medoid, PQ training and exact kNN on the GPU.
#include <algorithm>
#include <cmath>
#include <vector>

#include "dg_index.h"
#include "dg_search.cuh"

namespace dg {

// ------------------------------------------------------------ row encoders
__global__ void k_bf16(const float *v, uint64_t total, uint16_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = __bfloat16_as_ushort(__float2bfloat16_rn(v[i]));
}
__global__ void k_f16(const float *v, uint64_t total, uint16_t *out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = __half_as_ushort(__float2half_rn(v[i]));
}
// Int8Quantizer::encode (src/sq.rs:208-220)
__global__ void k_int8(const float *v, uint64_t n, uint32_t d, uint32_t dpad, float inv, float beta,
                       uint8_t *out, uint32_t stride) {
  const uint64_t total = n * stride;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / stride;
    const uint32_t c = (uint32_t)(i % stride);
    out[i] = c < d ? int8_code(v[r * dpad + c], inv, beta) : 0;
  }
}
// FP8 rows: per vector s = max|x| / 448 (1 for a zero vector), codes
// e4m3(x / s) rounded to nearest even with saturation, and |s * e4m3(x / s)|^2
// summed in coordinate order.  One thread per vector.
__global__ void k_fp8(const float *v, uint64_t n, uint32_t d, uint32_t dpad, uint8_t *codes, float2 *sn) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const float *x = v + r * dpad;
    float mx = 0.0f;
    for (uint32_t i = 0; i < d; ++i) mx = fmaxf(mx, fabsf(x[i]));
    const float s = mx > 0.0f ? __fdiv_rn(mx, 448.0f) : 1.0f;
    uint8_t *c = codes + r * dpad;
    float nn = 0.0f;
    for (uint32_t i = 0; i < dpad; ++i) {
      const __nv_fp8_storage_t e = i < d ? __nv_cvt_float_to_fp8(__fdiv_rn(x[i], s), __NV_SATFINITE, __NV_E4M3) : 0;
      c[i] = e;
      const float xv = __fmul_rn(s, __half2float(__half(__nv_cvt_fp8_to_halfraw(e, __NV_E4M3))));
      nn = __fadd_rn(nn, __fmul_rn(xv, xv));
    }
    sn[r] = make_float2(s, nn);
  }
}
// Sum of squared codes of every int8 row (padding bytes are zero).
__global__ void k_int8_norm(const uint8_t *codes, uint64_t n, uint32_t stride, uint32_t *out, uint32_t *sums) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 *row = reinterpret_cast<const uint4 *>(codes + r * stride);
    uint32_t s = 0, t = 0;
    for (uint32_t c = 0; c < stride / 16; ++c) {
      const uint4 v = row[c];
      s = __dp4a(v.x, v.x, s);
      s = __dp4a(v.y, v.y, s);
      s = __dp4a(v.z, v.z, s);
      s = __dp4a(v.w, v.w, s);
      t = __dp4a(v.x, 0x01010101u, t);
      t = __dp4a(v.y, 0x01010101u, t);
      t = __dp4a(v.z, 0x01010101u, t);
      t = __dp4a(v.w, 0x01010101u, t);
    }
    out[r] = s;
    if (sums) sums[r] = t;
  }
}
// ProductQuantizer::encode (src/pq.rs:122-149): argmin with strict '<'.
__global__ void k_pq_encode(const float *v, uint64_t n, uint32_t dpad, uint32_t M, uint32_t K,
                            uint32_t ds, const float *cb, uint8_t *codes, uint32_t stride) {
  const uint32_t m = blockIdx.y;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float *sub = v + i * dpad + m * ds;
    float best = 3.402823466e38f;
    uint32_t bc = 0;
    for (uint32_t c = 0; c < K; ++c) {
      const float *cen = cb + ((size_t)m * K + c) * ds;
      float acc = 0.0f;
      for (uint32_t j = 0; j < ds; ++j) {
        float t = __fsub_rn(sub[j], __ldg(cen + j));
        acc = __fadd_rn(acc, __fmul_rn(t, t));
      }
      if (acc < best) {
        best = acc;
        bc = c;
      }
    }
    codes[i * stride + m] = (uint8_t)bc;
  }
}

// RaBitQ encode_with (src/rabitq.rs:136-149,240-256), one warp per vector.
__global__ void k_rabitq_encode(const float *v, uint64_t n, uint32_t d, uint32_t dpad, uint32_t P,
                                const float *cen, const float *signs, uint8_t *codes,
                                uint32_t stride) {
  extern __shared__ __align__(16) float rbuf[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *r = rbuf + (size_t)warp * P;
  const uint64_t gw = blockIdx.x * (uint64_t)(blockDim.x >> 5) + warp;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t row = gw; row < n; row += nw) {
    const float *x = v + row * dpad;
    for (uint32_t i = lane; i < P; i += 32) r[i] = i < d ? __fsub_rn(x[i], cen[i]) : 0.0f;
    __syncwarp();
    float s = 0.0f;
    if (lane == 0)
      for (uint32_t i = 0; i < P; ++i) s = __fadd_rn(s, __fmul_rn(r[i], r[i]));
    const float norm = __shfl_sync(kFull, __fsqrt_rn(s), 0);
    if (norm > 0.0f)
      for (uint32_t i = lane; i < P; i += 32) r[i] = __fdiv_rn(r[i], norm);
    __syncwarp();
    for (int rd = 0; rd < 3; ++rd) {
      for (uint32_t i = lane; i < P; i += 32) r[i] = __fmul_rn(r[i], signs[rd * P + i]);
      __syncwarp();
      for (uint32_t h = 1; h < P; h *= 2) {
        for (uint32_t t = lane; t < P / 2; t += 32) {
          const uint32_t j = (t / h) * 2 * h + (t % h);
          const float a = r[j], b = r[j + h];
          r[j] = __fadd_rn(a, b);
          r[j + h] = __fsub_rn(a, b);
        }
        __syncwarp();
      }
    }
    uint8_t *code = codes + row * stride;
    for (uint32_t wd = 0; wd < P / 64; ++wd) {
      const bool b0 = r[wd * 64 + lane] > 0.0f, b1 = r[wd * 64 + 32 + lane] > 0.0f;
      const uint32_t lo = __ballot_sync(kFull, b0), hi = __ballot_sync(kFull, b1);
      if (lane == 0) {
        uint32_t *w = reinterpret_cast<uint32_t *>(code + wd * 8);
        w[0] = lo;
        w[1] = hi;
      }
    }
    if (lane == 0) {  // sequential sum of |x| in coordinate order, as the oracle
      float ip = 0.0f;
      for (uint32_t i = 0; i < P; ++i) ip = __fadd_rn(ip, fabsf(r[i]));
      ip = __fdiv_rn(ip, __fsqrt_rn((float)P));
      const float fac = ip > 0.0f ? __fdiv_rn(norm, ip) : 0.0f;
      float *tail = reinterpret_cast<float *>(code + P / 8);
      tail[0] = __fmul_rn(norm, norm);
      tail[1] = fac;
    }
    __syncwarp();
  }
}

// Squared norm of every decoded PQ code (ProductQuantizer::decode,
// src/pq.rs:151-160): the |x|^2 term of the cosine metric over codes, summed
// in coordinate order as angular() does.  One thread per vector.
__global__ void k_pq_dnorm2(const uint8_t *codes, uint64_t n, uint32_t stride, uint32_t M, uint32_t K,
                            uint32_t ds, const float *cb, float *out) {
  for (uint64_t row = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; row < n;
       row += (uint64_t)gridDim.x * blockDim.x) {
    const uint8_t *code = codes + row * stride;
    float bb = 0.0f;
    for (uint32_t m = 0; m < M; ++m) {
      const float *c = cb + ((size_t)m * K + code[m]) * ds;
      for (uint32_t j = 0; j < ds; ++j) bb = __fadd_rn(bb, __fmul_rn(c[j], c[j]));
    }
    out[row] = bb;
  }
}

// Squared norm of every decoded RaBitQ code (src/rabitq.rs:224-238): signs
// +-1/sqrt(P), three inverse rounds (Hadamard, then sign flip), then
// c + |v-c| * r over the first d coordinates, summed in coordinate order.
// One warp per vector.
__global__ void k_rq_dnorm2(const uint8_t *codes, uint64_t n, uint32_t stride, uint32_t d, uint32_t P,
                            const float *cen, const float *signs, float *out) {
  extern __shared__ __align__(16) float rbuf[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *r = rbuf + (size_t)warp * P;
  const uint64_t gw = blockIdx.x * (uint64_t)(blockDim.x >> 5) + warp;
  const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const float inv = __fdiv_rn(1.0f, __fsqrt_rn((float)P));
  for (uint64_t row = gw; row < n; row += nw) {
    const uint8_t *code = codes + row * stride;
    for (uint32_t i = lane; i < P; i += 32) r[i] = ((code[i >> 3] >> (i & 7)) & 1u) ? inv : -inv;
    __syncwarp();
    for (int rd = 2; rd >= 0; --rd) {
      for (uint32_t h = 1; h < P; h *= 2) {
        for (uint32_t t = lane; t < P / 2; t += 32) {
          const uint32_t j = (t / h) * 2 * h + (t % h);
          const float a = r[j], b = r[j + h];
          r[j] = __fadd_rn(a, b);
          r[j + h] = __fsub_rn(a, b);
        }
        __syncwarp();
      }
      for (uint32_t i = lane; i < P; i += 32) r[i] = __fmul_rn(r[i], signs[rd * P + i]);
      __syncwarp();
    }
    if (lane == 0) {
      const float norm = __fsqrt_rn(*reinterpret_cast<const float *>(code + P / 8));
      float bb = 0.0f;
      for (uint32_t i = 0; i < d; ++i) {
        const float o = __fadd_rn(cen[i], __fmul_rn(norm, r[i]));
        bb = __fadd_rn(bb, __fmul_rn(o, o));
      }
      out[row] = bb;
    }
    __syncwarp();
  }
}

__global__ void k_count(const uint64_t *labels, uint64_t n, uint32_t nf, const DgFilterOp *ops,
                        uint32_t nops, const uint64_t *pool, unsigned long long *count) {
  unsigned long long c = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    c += filter_eval(ops, nops, pool, labels + i * nf, nf) ? 1 : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

static int grid_for(uint64_t work, int threads) {
  uint64_t g = (work + threads - 1) / threads;
  return (int)std::min<uint64_t>(std::max<uint64_t>(g, 1), 148ull * 64);
}

// Squared norm of every BF16 row, summed in coordinate order in FP32.
__global__ void k_bf16_norms(const uint16_t *rows, uint64_t n, uint32_t dpad, float *out) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint16_t *x = rows + r * dpad;
    float s2 = 0.0f;
    for (uint32_t i = 0; i < dpad; ++i) {
      const float v = __uint_as_float((uint32_t)x[i] << 16);
      s2 = __fadd_rn(s2, __fmul_rn(v, v));
    }
    out[r] = s2;
  }
}

DgStatus encode_bf16_device(const float *vec, uint64_t n, uint32_t dpad, uint16_t *out, cudaStream_t st,
                            float *norms) {
  k_bf16<<<grid_for(n * dpad, 256), 256, 0, st>>>(vec, n * dpad, out);
  DG_CUDA(cudaGetLastError());
  if (norms) {
    k_bf16_norms<<<grid_for(n, 128), 128, 0, st>>>(out, n, dpad, norms);
    DG_CUDA(cudaGetLastError());
  }
  return DG_OK;
}
DgStatus encode_f16_device(const float *vec, uint64_t n, uint32_t dpad, uint16_t *out, cudaStream_t st) {
  k_f16<<<grid_for(n * dpad, 256), 256, 0, st>>>(vec, n * dpad, out);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus encode_int8_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, float scale,
                            float offset, uint8_t *codes, uint32_t stride, cudaStream_t st) {
  const float inv = 1.0f / scale;  // same f32 expressions as Int8Quantizer::encode
  const float beta = -offset / scale;
  k_int8<<<grid_for(n * stride, 256), 256, 0, st>>>(vec, n, d, dpad, inv, beta, codes, stride);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus encode_fp8_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, uint8_t *codes,
                           float2 *sn, cudaStream_t st) {
  k_fp8<<<grid_for(n, 128), 128, 0, st>>>(vec, n, d, dpad, codes, sn);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus int8_norms_device(const uint8_t *codes, uint64_t n, uint32_t stride, uint32_t *out, uint32_t *sums,
                           cudaStream_t st) {
  k_int8_norm<<<grid_for(n, 256), 256, 0, st>>>(codes, n, stride, out, sums);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus encode_pq_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, uint32_t M,
                          uint32_t K, const float *cb, uint8_t *codes, uint32_t stride,
                          cudaStream_t st) {
  dim3 grid((unsigned)std::min<uint64_t>((n + 127) / 128, 4096), M);
  k_pq_encode<<<grid, 128, 0, st>>>(vec, n, dpad, M, K, d / M, cb, codes, stride);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus encode_rabitq_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, uint32_t P,
                              const float *centroid, const float *signs, uint8_t *codes,
                              uint32_t stride, cudaStream_t st) {
  const int warps = 4;
  const size_t smem = (size_t)warps * P * 4;
  DG_CUDA(cudaFuncSetAttribute(k_rabitq_encode, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int blocks = (int)std::min<uint64_t>((n + warps - 1) / warps, 148ull * 16);
  k_rabitq_encode<<<blocks, warps * 32, smem, st>>>(vec, n, d, dpad, P, centroid, signs, codes, stride);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus decoded_norms_device(const DgIndex *idx, float *out, cudaStream_t st) {
  if (idx->quant == DG_Q_PQ) {
    k_pq_dnorm2<<<grid_for(idx->n, 128), 128, 0, st>>>(idx->codes, idx->n, idx->code_stride, idx->pq_M,
                                                       idx->pq_K, idx->d / idx->pq_M, idx->pq_cb, out);
  } else {
    const int warps = 4;
    const uint32_t P = idx->rq_padded;
    const size_t smem = (size_t)warps * P * 4;
    DG_CUDA(cudaFuncSetAttribute(k_rq_dnorm2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int blocks = (int)std::min<uint64_t>((idx->n + warps - 1) / warps, 148ull * 16);
    k_rq_dnorm2<<<blocks, warps * 32, smem, st>>>(idx->codes, idx->n, idx->code_stride, idx->d, P,
                                                  idx->rq_centroid, idx->rq_signs, out);
  }
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}
DgStatus count_matching_device(const uint64_t *labels, uint64_t n, uint32_t nf,
                               const DgFilterOp *ops, uint32_t nops, const uint64_t *pool,
                               unsigned long long *count, cudaStream_t st) {
  k_count<<<grid_for(n, 256), 256, 0, st>>>(labels, n, nf, ops, nops, pool, count);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

// ------------------------------------------------------------------ medoid
// calculate_medoid (src/lib.rs:748-768): centroid summed in f64 and rounded
// once to f32, f64 distances, lowest index on ties (same as the oracle).
__global__ void k_colsum(const float *v, uint64_t n, uint32_t d, uint32_t dpad, double *sums) {
  for (uint32_t c = threadIdx.x; c < d; c += blockDim.x) {
    double acc = 0.0;
    for (uint64_t r = blockIdx.x; r < n; r += gridDim.x) acc += (double)v[r * dpad + c];
    atomicAdd(sums + c, acc);
  }
}
__device__ __forceinline__ unsigned long long ordered_u64(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ double medoid_metric(const float *x, const float *c, uint32_t d, int metric) {
  if (metric == DG_L2SQ || metric == DG_L2) {
    double s = 0.0;
    for (uint32_t j = 0; j < d; ++j) {
      double t = __dsub_rn((double)c[j], (double)x[j]);
      s = __dadd_rn(s, __dmul_rn(t, t));
    }
    return s;
  }
  double ab = 0.0, aa = 0.0, bb = 0.0;
  for (uint32_t j = 0; j < d; ++j) {
    ab = __dadd_rn(ab, __dmul_rn((double)c[j], (double)x[j]));
    aa = __dadd_rn(aa, __dmul_rn((double)c[j], (double)c[j]));
    bb = __dadd_rn(bb, __dmul_rn((double)x[j], (double)x[j]));
  }
  if (metric == DG_COSINE) return (aa == 0.0 || bb == 0.0) ? 1.0 : 1.0 - ab / (sqrt(aa) * sqrt(bb));
  return 1.0 - ab;
}
__global__ void k_medoid_min(const float *v, uint64_t n, uint32_t d, uint32_t dpad, const float *c,
                             int metric, unsigned long long *best) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicMin(best, ordered_u64(medoid_metric(v + i * dpad, c, d, metric)));
}
__global__ void k_medoid_arg(const float *v, uint64_t n, uint32_t d, uint32_t dpad, const float *c,
                             int metric, const unsigned long long *best, unsigned long long *arg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (ordered_u64(medoid_metric(v + i * dpad, c, d, metric)) == *best) atomicMin(arg, (unsigned long long)i);
}

DgStatus medoid_device(const float *vec, uint64_t n, uint32_t d, uint32_t dpad, int metric,
                       uint32_t *out, cudaStream_t st) {
  double *sums = nullptr;
  float *cen = nullptr;
  unsigned long long *best = nullptr;
  DG_CUDA(cudaMallocAsync(&sums, d * 8, st));
  DG_CUDA(cudaMallocAsync(&cen, d * 4, st));
  DG_CUDA(cudaMallocAsync(&best, 16, st));
  DG_CUDA(cudaMemsetAsync(sums, 0, d * 8, st));
  k_colsum<<<(unsigned)std::min<uint64_t>(n, 1024), 128, 0, st>>>(vec, n, d, dpad, sums);
  std::vector<double> hs(d);
  DG_CUDA(cudaMemcpyAsync(hs.data(), sums, d * 8, cudaMemcpyDeviceToHost, st));
  DG_CUDA(cudaStreamSynchronize(st));
  std::vector<float> hc(d);
  for (uint32_t j = 0; j < d; ++j) hc[j] = (float)(hs[j] / (double)n);
  DG_CUDA(cudaMemcpyAsync(cen, hc.data(), d * 4, cudaMemcpyHostToDevice, st));
  unsigned long long init[2] = {~0ull, ~0ull};
  DG_CUDA(cudaMemcpyAsync(best, init, 16, cudaMemcpyHostToDevice, st));
  k_medoid_min<<<grid_for(n, 256), 256, 0, st>>>(vec, n, d, dpad, cen, metric, best);
  k_medoid_arg<<<grid_for(n, 256), 256, 0, st>>>(vec, n, d, dpad, cen, metric, best, best + 1);
  unsigned long long res[2];
  DG_CUDA(cudaMemcpyAsync(res, best, 16, cudaMemcpyDeviceToHost, st));
  DG_CUDA(cudaStreamSynchronize(st));
  cudaFreeAsync(sums, st);
  cudaFreeAsync(cen, st);
  cudaFreeAsync(best, st);
  *out = (uint32_t)res[1];
  return DG_OK;
}

// -------------------------------------------------------------- exact kNN
// Brute force with FP64 accumulation.  A block holds 8 queries (one per
// warp); base rows stream through shared memory 32 at a time and each warp
// keeps its k best (distance, id) keys with the same merge as the search.
constexpr int kKnnWarps = 8;
__global__ void __launch_bounds__(256) k_exact_knn(const float *X, uint64_t n, uint32_t d, uint32_t dpad,
                                                   const float *Q, uint32_t nq, uint32_t k, int metric,
                                                   uint32_t kcap, uint32_t *out_ids, float *out_d) {
  extern __shared__ __align__(16) uint8_t sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rs = d + 1;  // padded row stride (bank-conflict free)
  float *tile = reinterpret_cast<float *>(sm);
  float *qsm = tile + 32 * rs;
  uint64_t *lists = reinterpret_cast<uint64_t *>(sm + align16((32 * rs + kKnnWarps * d) * 4));
  uint64_t *L0 = lists + (size_t)warp * (2 * kcap + 32);
  uint64_t *L1 = L0 + kcap;
  uint64_t *cst = L1 + kcap;
  const uint32_t q = blockIdx.x * kKnnWarps + warp;
  const bool active = q < nq;
  for (uint32_t j = lane; j < d; j += 32) qsm[warp * d + j] = active ? Q[(size_t)q * d + j] : 0.0f;
  double qq = 0.0;
  for (uint32_t j = 0; j < d; ++j) qq += (double)qsm[warp * d + j] * (double)qsm[warp * d + j];
  int size = 0, cur = 0;
  uint64_t *Ls[2] = {L0, L1};
  for (uint64_t base = 0; base < n; base += 32) {
    __syncthreads();
    const uint32_t rows = (uint32_t)((n - base) < 32 ? (n - base) : 32);
    for (uint32_t e = threadIdx.x; e < rows * d; e += blockDim.x) {
      const uint32_t r = e / d, c = e % d;
      tile[r * rs + c] = X[(base + r) * dpad + c];
    }
    __syncthreads();
    if (!active) continue;
    uint64_t key = kKeyInvalid;
    if ((uint32_t)lane < rows) {
      const float *x = tile + lane * rs;
      const float *qv = qsm + warp * d;
      double v;
      if (metric == DG_L2SQ || metric == DG_L2) {
        double s = 0.0;
        for (uint32_t j = 0; j < d; ++j) {
          double t = (double)qv[j] - (double)x[j];
          s = fma(t, t, s);
        }
        v = metric == DG_L2 ? sqrt(s) : s;
      } else {
        double ab = 0.0, bb = 0.0;
        for (uint32_t j = 0; j < d; ++j) {
          ab = fma((double)qv[j], (double)x[j], ab);
          bb = fma((double)x[j], (double)x[j], bb);
        }
        v = metric == DG_COSINE ? ((qq == 0.0 || bb == 0.0) ? 1.0 : 1.0 - ab / (sqrt(qq) * sqrt(bb)))
                                : 1.0 - ab;
      }
      key = make_key((float)v, (uint32_t)(base + lane));
    }
    // skip the merge when no lane beats the current k-th
    const bool maybe = key != kKeyInvalid && (size < (int)k || key < Ls[cur][k - 1]);
    if (!__any_sync(kFull, maybe)) continue;
    const int nc = prepare_batch(key, Ls[cur], size, (int)k, cst, lane);
    if (nc > 0) {
      size = merge_keys(Ls[cur], size, Ls[cur ^ 1], (int)k, cst, nc, lane);
      cur ^= 1;
    }
  }
  if (!active) return;
  for (int i = lane; i < (int)k; i += 32) {
    out_ids[(size_t)q * k + i] = i < size ? key_id(Ls[cur][i]) : DG_PAD;
    out_d[(size_t)q * k + i] = i < size ? key_dist(Ls[cur][i]) : __int_as_float(0x7f800000);
  }
}

// ------------------------------------------------------------ PQ training
// ProductQuantizer::train (src/pq.rs:51-119): per subspace, k-means++ seeding
// then Lloyd iterations; empty clusters restart from a random training point.
__global__ void k_mindist_update(const float *S, uint32_t ns, uint32_t d, uint32_t M, uint32_t ds,
                                 const float *cb, uint32_t K, uint32_t c_new, float *mind) {
  const uint32_t m = blockIdx.y;
  const float *cen = cb + ((size_t)m * K + c_new) * ds;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    const float *x = S + (size_t)i * d + m * ds;
    float acc = 0.0f;
    for (uint32_t j = 0; j < ds; ++j) {
      float t = __fsub_rn(x[j], cen[j]);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    }
    float &md = mind[(size_t)m * ns + i];
    md = fminf(md, acc);
  }
}
// One block per subspace: D^2-weighted draw of the next seed.
__global__ void k_pick_next(const float *S, uint32_t ns, uint32_t d, uint32_t ds, float *cb, uint32_t K,
                            uint32_t c_new, const float *mind, uint64_t seed) {
  __shared__ double part[1024];
  __shared__ uint32_t chosen;
  const uint32_t m = blockIdx.x;
  const float *md = mind + (size_t)m * ns;
  const uint32_t per = (ns + blockDim.x - 1) / blockDim.x;
  const uint32_t lo = threadIdx.x * per, hi = min(ns, lo + per);
  double s = 0.0;
  for (uint32_t i = lo; i < hi; ++i) s += md[i];
  part[threadIdx.x] = s;
  if (threadIdx.x == 0) chosen = ns - 1;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (uint32_t t = 0; t < blockDim.x; ++t) tot += part[t];
    const double u = (double)(rand4(seed, 0x6b6d, m, c_new) >> 11) * (1.0 / 9007199254740992.0);
    if (tot <= 0.0) {
      chosen = (uint32_t)range_of(rand4(seed, 0x6b6e, m, c_new), ns);
    } else {
      const double thr = u * tot;
      double cum = 0.0;
      for (uint32_t t = 0; t < blockDim.x; ++t) {
        if (cum + part[t] >= thr) {
          const uint32_t a = t * per, b = min(ns, a + per);
          for (uint32_t i = a; i < b; ++i) {
            cum += md[i];
            if (cum >= thr) {
              chosen = i;
              break;
            }
          }
          break;
        }
        cum += part[t];
      }
    }
  }
  __syncthreads();
  for (uint32_t j = threadIdx.x; j < ds; j += blockDim.x)
    cb[((size_t)m * K + c_new) * ds + j] = S[(size_t)chosen * d + m * ds + j];
}
__global__ void k_assign_accum(const float *S, uint32_t ns, uint32_t d, uint32_t ds, const float *cb,
                               uint32_t K, double *sums, unsigned int *counts) {
  const uint32_t m = blockIdx.y;
  extern __shared__ float cbs[];
  for (uint32_t e = threadIdx.x; e < K * ds; e += blockDim.x) cbs[e] = cb[(size_t)m * K * ds + e];
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    const float *x = S + (size_t)i * d + m * ds;
    float best = 3.402823466e38f;
    uint32_t bc = 0;
    for (uint32_t c = 0; c < K; ++c) {
      float acc = 0.0f;
      for (uint32_t j = 0; j < ds; ++j) {
        float t = __fsub_rn(x[j], cbs[c * ds + j]);
        acc = __fadd_rn(acc, __fmul_rn(t, t));
      }
      if (acc < best) {
        best = acc;
        bc = c;
      }
    }
    atomicAdd(counts + (size_t)m * K + bc, 1u);
    for (uint32_t j = 0; j < ds; ++j) atomicAdd(sums + ((size_t)m * K + bc) * ds + j, (double)x[j]);
  }
}
__global__ void k_update(const float *S, uint32_t ns, uint32_t d, uint32_t M, uint32_t ds, float *cb,
                         uint32_t K, const double *sums, const unsigned int *counts, uint64_t seed,
                         uint32_t iter) {
  const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= M * K) return;
  const uint32_t m = e / K, c = e % K;
  const unsigned int cnt = counts[e];
  if (cnt > 0) {
    for (uint32_t j = 0; j < ds; ++j) cb[(size_t)e * ds + j] = (float)(sums[(size_t)e * ds + j] / (double)cnt);
  } else {
    const uint32_t r = (uint32_t)range_of(rand4(seed, 0x6b6f + iter, m, c), ns);
    for (uint32_t j = 0; j < ds; ++j) cb[(size_t)e * ds + j] = S[(size_t)r * d + m * ds + j];
  }
}

}  // namespace dg

using namespace dg;

extern "C" {

DgStatus dg_medoid(const float *X, uint64_t n, uint32_t dim, int32_t metric, int32_t device,
                   uint32_t *out_medoid) {
  if (!X || !out_medoid || n == 0 || dim == 0) return fail(DG_EINVAL, "bad medoid arguments");
  DG_CUDA(cudaSetDevice(device));
  const uint32_t dpad = dpad_of(dim);
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float *v = nullptr;
  DgStatus s = DG_OK;
  if (cudaMallocAsync(&v, n * dpad * 4, st) != cudaSuccess) s = fail(DG_ENOMEM, "medoid staging");
  if (s == DG_OK) s = upload_rows_f32(X, n, dim, dpad, v, st);
  if (s == DG_OK) s = medoid_device(v, n, dim, dpad, metric, out_medoid, st);
  if (v) cudaFreeAsync(v, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}

DgStatus dg_fp8_encode(const float *X, uint64_t n, uint32_t dim, int32_t device, uint8_t *out_codes,
                       float *out_scales) {
  if (!X || !out_codes || !out_scales) return fail(DG_EINVAL, "null argument");
  if (n == 0 || dim == 0) return DG_OK;
  DG_CUDA(cudaSetDevice(device));
  const uint32_t dpad = dpad_of(dim);
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float *v = nullptr;
  uint8_t *codes = nullptr;
  float2 *sn = nullptr;
  DgStatus s = DG_OK;
  if (cudaMallocAsync(&v, n * dpad * 4, st) != cudaSuccess || cudaMallocAsync(&codes, n * dpad, st) != cudaSuccess ||
      cudaMallocAsync(&sn, n * sizeof(float2), st) != cudaSuccess)
    s = fail(DG_ENOMEM, "fp8 encode staging");
  if (s == DG_OK) s = upload_rows_f32(X, n, dim, dpad, v, st);
  if (s == DG_OK) s = encode_fp8_device(v, n, dim, dpad, codes, sn, st);
  if (s == DG_OK && cudaMemcpy2DAsync(out_codes, dim, codes, dpad, dim, n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    s = fail(DG_EDEVICE, "code download");
  if (s == DG_OK && cudaMemcpy2DAsync(out_scales, 4, sn, sizeof(float2), 4, n, cudaMemcpyDeviceToHost, st) !=
                        cudaSuccess)
    s = fail(DG_EDEVICE, "scale download");
  cudaStreamSynchronize(st);
  if (v) cudaFreeAsync(v, st);
  if (codes) cudaFreeAsync(codes, st);
  if (sn) cudaFreeAsync(sn, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}

DgStatus dg_pq_encode(const float *X, uint64_t n, uint32_t dim, uint32_t M, uint32_t K,
                      const float *codebooks, int32_t device, uint8_t *out_codes) {
  if (!X || !codebooks || !out_codes) return fail(DG_EINVAL, "null argument");
  if (M == 0 || dim % M) return fail(DG_EINVAL, "dimension not divisible by num_subspaces");
  if (K == 0 || K > 256) return fail(DG_EINVAL, "num_centroids must be in [1, 256]");
  DG_CUDA(cudaSetDevice(device));
  const uint32_t dpad = dpad_of(dim);
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float *v = nullptr, *cb = nullptr;
  uint8_t *codes = nullptr;
  DgStatus s = DG_OK;
  const size_t cbb = (size_t)M * K * (dim / M) * 4;
  if (cudaMallocAsync(&v, n * dpad * 4, st) != cudaSuccess || cudaMallocAsync(&cb, cbb, st) != cudaSuccess ||
      cudaMallocAsync(&codes, n * M, st) != cudaSuccess)
    s = fail(DG_ENOMEM, "pq encode staging");
  if (s == DG_OK) s = upload_rows_f32(X, n, dim, dpad, v, st);
  if (s == DG_OK && cudaMemcpyAsync(cb, codebooks, cbb, cudaMemcpyHostToDevice, st) != cudaSuccess)
    s = fail(DG_EDEVICE, "codebook upload");
  if (s == DG_OK) s = encode_pq_device(v, n, dim, dpad, M, K, cb, codes, M, st);
  if (s == DG_OK && cudaMemcpyAsync(out_codes, codes, n * M, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    s = fail(DG_EDEVICE, "code download");
  cudaStreamSynchronize(st);
  if (v) cudaFreeAsync(v, st);
  if (cb) cudaFreeAsync(cb, st);
  if (codes) cudaFreeAsync(codes, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}

DgStatus dg_rabitq_encode(const float *X, uint64_t n, uint32_t dim, uint32_t padded, const float *centroid,
                          const float *signs, int32_t device, uint8_t *out_codes) {
  if (!X || !centroid || !signs || !out_codes) return fail(DG_EINVAL, "null argument");
  if (padded < 64 || (padded & (padded - 1)) || padded < dim) return fail(DG_EINVAL, "bad padded dimension");
  if (n == 0) return DG_OK;
  DG_CUDA(cudaSetDevice(device));
  const uint32_t dpad = dpad_of(dim), cs = padded / 8 + 8;
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float *v = nullptr, *cen = nullptr, *sg = nullptr;
  uint8_t *codes = nullptr;
  DgStatus s = DG_OK;
  if (cudaMallocAsync(&v, n * dpad * 4, st) != cudaSuccess || cudaMallocAsync(&cen, (size_t)dim * 4, st) != cudaSuccess ||
      cudaMallocAsync(&sg, (size_t)3 * padded * 4, st) != cudaSuccess ||
      cudaMallocAsync(&codes, n * cs, st) != cudaSuccess)
    s = fail(DG_ENOMEM, "rabitq encode staging");
  if (s == DG_OK) s = upload_rows_f32(X, n, dim, dpad, v, st);
  if (s == DG_OK && (cudaMemcpyAsync(cen, centroid, (size_t)dim * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                     cudaMemcpyAsync(sg, signs, (size_t)3 * padded * 4, cudaMemcpyHostToDevice, st) != cudaSuccess))
    s = fail(DG_EDEVICE, "rabitq parameter upload");
  if (s == DG_OK) s = encode_rabitq_device(v, n, dim, dpad, padded, cen, sg, codes, cs, st);
  if (s == DG_OK && cudaMemcpyAsync(out_codes, codes, n * cs, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    s = fail(DG_EDEVICE, "code download");
  cudaStreamSynchronize(st);
  for (void *p : {(void *)v, (void *)cen, (void *)sg, (void *)codes})
    if (p) cudaFreeAsync(p, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}

DgStatus dg_pq_train(const float *X, uint64_t n, uint32_t dim, uint32_t M, uint32_t K,
                     uint32_t iterations, uint64_t sample, uint64_t seed, int32_t device,
                     float *out_codebooks) {
  if (!X || !out_codebooks || n == 0) return fail(DG_EINVAL, "No vectors to train on");
  if (K > 256) return fail(DG_EINVAL, "num_centroids " + std::to_string(K) + " exceeds 256 (codes are u8)");
  if (M == 0 || dim % M)
    return fail(DG_EINVAL, "Dimension " + std::to_string(dim) + " not divisible by num_subspaces " +
                               std::to_string(M));
  if (K == 0) return fail(DG_EINVAL, "num_centroids must be >= 1");
  DG_CUDA(cudaSetDevice(device));
  const uint32_t ds = dim / M;
  // training sample (src/pq.rs:75-82): `sample` distinct rows drawn by a
  // seeded partial Fisher-Yates shuffle when the set is larger
  std::vector<uint64_t> rows;
  if (sample > 0 && n > sample) {
    std::vector<uint64_t> perm(n);
    for (uint64_t i = 0; i < n; ++i) perm[i] = i;
    for (uint64_t i = 0; i < sample; ++i) {
      uint64_t j = i + (uint64_t)(((unsigned __int128)rand4(seed, 0x7371, i, 0) * (n - i)) >> 64);
      std::swap(perm[i], perm[j]);
    }
    rows.assign(perm.begin(), perm.begin() + sample);
  } else {
    rows.resize(n);
    for (uint64_t i = 0; i < n; ++i) rows[i] = i;
  }
  const uint32_t ns = (uint32_t)rows.size();
  std::vector<float> hs((size_t)ns * dim);
  for (uint32_t i = 0; i < ns; ++i) std::copy(X + rows[i] * dim, X + rows[i] * dim + dim, hs.begin() + (size_t)i * dim);
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float *S = nullptr, *cb = nullptr, *mind = nullptr;
  double *sums = nullptr;
  unsigned int *counts = nullptr;
  DgStatus s = DG_OK;
  const size_t cbn = (size_t)M * K * ds;
  if (cudaMallocAsync(&S, hs.size() * 4, st) != cudaSuccess || cudaMallocAsync(&cb, cbn * 4, st) != cudaSuccess ||
      cudaMallocAsync(&mind, (size_t)M * ns * 4, st) != cudaSuccess ||
      cudaMallocAsync(&sums, cbn * 8, st) != cudaSuccess ||
      cudaMallocAsync(&counts, (size_t)M * K * 4, st) != cudaSuccess)
    s = fail(DG_ENOMEM, "pq training staging");
  if (s == DG_OK) {
    cudaMemcpyAsync(S, hs.data(), hs.size() * 4, cudaMemcpyHostToDevice, st);
    // k-means++ seeding (src/pq.rs:301-341)
    std::vector<float> inf((size_t)M * ns, 3.402823466e38f);
    cudaMemcpyAsync(mind, inf.data(), inf.size() * 4, cudaMemcpyHostToDevice, st);
    const uint32_t keff = std::min<uint32_t>(K, ns);
    std::vector<float> hcb(cbn);
    for (uint32_t m = 0; m < M; ++m) {
      const uint32_t first = (uint32_t)(((unsigned __int128)rand4(seed, 0x6b6c, m, 0) * ns) >> 64);
      std::copy(hs.begin() + (size_t)first * dim + m * ds, hs.begin() + (size_t)first * dim + m * ds + ds,
                hcb.begin() + (size_t)m * K * ds);
    }
    cudaMemcpyAsync(cb, hcb.data(), cbn * 4, cudaMemcpyHostToDevice, st);
    dim3 g((ns + 255) / 256, M);
    for (uint32_t c = 1; c < keff; ++c) {
      k_mindist_update<<<g, 256, 0, st>>>(S, ns, dim, M, ds, cb, K, c - 1, mind);
      k_pick_next<<<M, 1024, 0, st>>>(S, ns, dim, ds, cb, K, c, mind, seed);
    }
    // replicate when K exceeds the sample (src/pq.rs:344-350)
    if (keff < K) {
      cudaMemcpyAsync(hcb.data(), cb, cbn * 4, cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      for (uint32_t m = 0; m < M; ++m)
        for (uint32_t c = keff; c < K; ++c)
          std::copy(hcb.begin() + ((size_t)m * K + c % keff) * ds, hcb.begin() + ((size_t)m * K + c % keff) * ds + ds,
                    hcb.begin() + ((size_t)m * K + c) * ds);
      cudaMemcpyAsync(cb, hcb.data(), cbn * 4, cudaMemcpyHostToDevice, st);
    }
    // Lloyd iterations (src/pq.rs:353-408)
    const size_t smem = (size_t)K * ds * 4;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_assign_accum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    for (uint32_t it = 0; it < iterations; ++it) {
      cudaMemsetAsync(sums, 0, cbn * 8, st);
      cudaMemsetAsync(counts, 0, (size_t)M * K * 4, st);
      dim3 ga((unsigned)std::min<uint32_t>((ns + 255) / 256, 256), M);
      k_assign_accum<<<ga, 256, smem, st>>>(S, ns, dim, ds, cb, K, sums, counts);
      k_update<<<(M * K + 255) / 256, 256, 0, st>>>(S, ns, dim, M, ds, cb, K, sums, counts, seed, it);
    }
    if (cudaMemcpyAsync(out_codebooks, cb, cbn * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
      s = fail(DG_EDEVICE, "codebook download");
    if (cudaStreamSynchronize(st) != cudaSuccess) s = fail(DG_EDEVICE, cudaGetErrorString(cudaGetLastError()));
  }
  if (S) cudaFreeAsync(S, st);
  if (cb) cudaFreeAsync(cb, st);
  if (mind) cudaFreeAsync(mind, st);
  if (sums) cudaFreeAsync(sums, st);
  if (counts) cudaFreeAsync(counts, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}

DgStatus dg_exact_knn(const float *X, uint64_t n, uint32_t dim, const float *Q, uint32_t nq,
                      uint32_t k, int32_t metric, int32_t device, uint32_t *out_ids,
                      float *out_dists) {
  if (!X || !Q || !out_ids || !out_dists || n == 0 || dim == 0) return fail(DG_EINVAL, "bad arguments");
  if (k == 0 || k > 1024) return fail(DG_EINVAL, "k must be in [1, 1024]");
  DG_CUDA(cudaSetDevice(device));
  const uint32_t dpad = dpad_of(dim);
  cudaStream_t st;
  DG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  float *v = nullptr, *q = nullptr, *od = nullptr;
  uint32_t *oi = nullptr;
  DgStatus s = DG_OK;
  if (cudaMallocAsync(&v, n * dpad * 4, st) != cudaSuccess || cudaMallocAsync(&q, (size_t)nq * dim * 4, st) != cudaSuccess ||
      cudaMallocAsync(&oi, (size_t)nq * k * 4, st) != cudaSuccess ||
      cudaMallocAsync(&od, (size_t)nq * k * 4, st) != cudaSuccess)
    s = fail(DG_ENOMEM, "exact knn staging");
  if (s == DG_OK) s = upload_rows_f32(X, n, dim, dpad, v, st);
  if (s == DG_OK) cudaMemcpyAsync(q, Q, (size_t)nq * dim * 4, cudaMemcpyHostToDevice, st);
  if (s == DG_OK) {
    uint32_t kcap = 32;
    while (kcap < k) kcap <<= 1;
    const size_t smem = align16((32 * (dim + 1) + kKnnWarps * dim) * 4) + (size_t)kKnnWarps * (2 * kcap + 32) * 8;
    if (cudaFuncSetAttribute(k_exact_knn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      s = fail(DG_ENOTSUP, "exact knn tile does not fit in shared memory");
    if (s == DG_OK) {
      k_exact_knn<<<(nq + kKnnWarps - 1) / kKnnWarps, 256, smem, st>>>(v, n, dim, dpad, q, nq, k, metric, kcap, oi, od);
      if (cudaGetLastError() != cudaSuccess) s = fail(DG_EDEVICE, "exact knn launch");
    }
  }
  if (s == DG_OK) {
    cudaMemcpyAsync(out_ids, oi, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(out_dists, od, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) s = fail(DG_EDEVICE, "exact knn failed");
  }
  if (v) cudaFreeAsync(v, st);
  if (q) cudaFreeAsync(q, st);
  if (oi) cudaFreeAsync(oi, st);
  if (od) cudaFreeAsync(od, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return s;
}

}  // extern "C"
