// dg_schedule.cu -- locality-aware order of a batch's queries.
//
// A batch's queries are searched by a persistent grid that hands them out in
// order.  Queries near one another in space traverse the same region of the
// graph and read the same rows; when they run at the same time those rows
// are served by L2 instead of DRAM.  This orders a batch by each query's
// nearest of P pivot rows (rows of the index spread evenly over its ids): a
// counting sort of the queries by pivot, whose positions the search kernel
// maps back to query ids (results are written at each query's own row, so
// the order never changes a result).  dg_index_autotune decides per kind of
// search whether the order pays for its three small kernels.
#include <algorithm>

#include "dg_index.h"

namespace dg {

// Each thread scores one query against every pivot (pivots staged in shared
// memory, read as broadcasts), keeps the nearest and counts it.
template <int P>
__global__ void __launch_bounds__(128) k_pivot_assign(const float *__restrict__ Q, uint32_t nq, uint32_t d,
                                                      const float *__restrict__ piv, uint32_t dpad, uint32_t *bin,
                                                      uint32_t *hist) {
  extern __shared__ float sp[];  // [d][P]: dimension-major, so a step reads P consecutive floats
  for (uint32_t t = threadIdx.x; t < (uint32_t)P * d; t += blockDim.x) {
    const uint32_t p = t % P, i = t / P;
    sp[t] = piv[(size_t)p * dpad + i];
  }
  __syncthreads();
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
    float acc[P];
#pragma unroll
    for (int p = 0; p < P; ++p) acc[p] = 0.0f;
    const float *qr = Q + (size_t)q * d;
    for (uint32_t i = 0; i < d; ++i) {
      const float qi = __ldg(qr + i);
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const float t = qi - sp[i * P + p];
        acc[p] = fmaf(t, t, acc[p]);
      }
    }
    uint32_t best = 0;
#pragma unroll
    for (int p = 1; p < P; ++p)
      if (acc[p] < acc[best]) best = p;
    bin[q] = best;
    atomicAdd(hist + best, 1u);
  }
}

// Exclusive scan of the P bin counts (one block of P threads, P <= 1024).
__global__ void k_pivot_scan(uint32_t *hist, uint32_t P) {
  __shared__ uint32_t s[1024];
  const uint32_t t = threadIdx.x;
  s[t] = t < P ? hist[t] : 0u;
  __syncthreads();
  for (uint32_t o = 1; o < blockDim.x; o <<= 1) {
    const uint32_t v = t >= o ? s[t - o] : 0u;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  if (t < P) hist[t] = s[t] - (t < P ? hist[t] : 0u);
}

__global__ void k_pivot_scatter(const uint32_t *bin, uint32_t nq, uint32_t *offs, uint32_t *perm) {
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x)
    perm[atomicAdd(offs + bin[q], 1u)] = q;
}

uint32_t pivot_count(uint32_t dpad) {
  // the pivots fill at most 32 KB of shared memory
  const uint32_t p = 32768u / (dpad * 4u);
  return p >= 32 ? 32 : p >= 16 ? 16 : 8;
}

DgStatus ensure_pivots(DgIndex *idx) {
  if (idx->pivots) return DG_OK;
  const uint32_t P = pivot_count(idx->dpad);
  DgStatus s = dev_alloc(idx, (void **)&idx->pivots, (size_t)P * idx->dpad * 4);
  if (s != DG_OK) return s;
  for (uint32_t p = 0; p < P; ++p) {
    const uint64_t row = (uint64_t)p * idx->n / P;
    DG_CUDA(cudaMemcpyAsync(idx->pivots + (size_t)p * idx->dpad, idx->vec + row * idx->dpad, idx->dpad * 4,
                            cudaMemcpyDeviceToDevice, idx->stream));
  }
  DG_CUDA(cudaStreamSynchronize(idx->stream));
  idx->npiv = P;
  return DG_OK;
}

DgStatus order_queries(const DgIndex *idx, const float *Q, uint32_t nq, uint32_t *perm, uint32_t *bin,
                       uint32_t *hist, cudaStream_t st) {
  const uint32_t P = idx->npiv, d = idx->d;
  DG_CUDA(cudaMemsetAsync(hist, 0, P * 4, st));
  const uint32_t threads = 128, grid = std::max(1u, std::min((nq + threads - 1) / threads, 148u * 8u));
  const size_t smem = (size_t)P * d * 4;
  switch (P) {
    case 32: k_pivot_assign<32><<<grid, threads, smem, st>>>(Q, nq, d, idx->pivots, idx->dpad, bin, hist); break;
    case 16: k_pivot_assign<16><<<grid, threads, smem, st>>>(Q, nq, d, idx->pivots, idx->dpad, bin, hist); break;
    default: k_pivot_assign<8><<<grid, threads, smem, st>>>(Q, nq, d, idx->pivots, idx->dpad, bin, hist); break;
  }
  k_pivot_scan<<<1, 1024, 0, st>>>(hist, P);
  k_pivot_scatter<<<grid, threads, 0, st>>>(bin, nq, hist, perm);
  DG_CUDA(cudaGetLastError());
  return DG_OK;
}

}  // namespace dg
