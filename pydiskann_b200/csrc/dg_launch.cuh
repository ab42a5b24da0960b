// dg_launch.cuh -- host-side launch of the beam-search kernel instantiations.
#pragma once
#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "dg_search_kernel.cuh"

namespace dg {

struct LaunchInfo {
  int grid = 0;
  int blocks_per_sm = 0;
  uint32_t smem = 0;
};

// Launch geometry: 4 warps per block (or the schedule's 2 or 1), as many
// resident blocks as shared memory and registers allow on every SM, never more
// warps than queries.
// Resident blocks per SM of (device, kernel, shared-memory size), and the
// largest dynamic shared memory already granted to (device, kernel): the
// attribute and occupancy queries run once, not on every launch (a serving
// loop launches thousands of small batches per second).
struct LaunchGeometry {
  std::mutex mu;
  std::unordered_map<const void *, int> sms, optin;                  // per device (key: device id)
  std::unordered_map<uint64_t, int> granted;                           // (device, kernel) -> smem
  std::unordered_map<uint64_t, std::unordered_map<uint32_t, int>> nb;  // (device, kernel) -> smem -> blocks
};
inline LaunchGeometry &launch_geometry() {
  static LaunchGeometry g;
  return g;
}

template <typename K>
DgStatus launch_persistent(K kernel, const SearchArgs &a, const WarpLayout &Ly, cudaStream_t st,
                           LaunchInfo *info) {
  const uint32_t wpb = (a.wpb == 1 || a.wpb == 2) ? a.wpb : 4u;  // warps per CTA
  const uint32_t smem = Ly.total * wpb;
  int dev = 0;
  DG_CUDA(cudaGetDevice(&dev));
  LaunchGeometry &G = launch_geometry();
  const void *kp = reinterpret_cast<const void *>(kernel);
  const uint64_t key = (reinterpret_cast<uint64_t>(kp) << 8) ^ (uint64_t)dev;
  const void *dkey = reinterpret_cast<const void *>((uintptr_t)dev + 1);
  int sms = 0, nb = 0;
  {
    std::lock_guard<std::mutex> lk(G.mu);
    auto s_it = G.sms.find(dkey);
    if (s_it == G.sms.end()) {
      int m = 0, o = 0;
      DG_CUDA(cudaDeviceGetAttribute(&o, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
      DG_CUDA(cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev));
      G.optin[dkey] = o;
      s_it = G.sms.emplace(dkey, m).first;
    }
    sms = s_it->second;
    if (smem > (uint32_t)G.optin[dkey])
      return fail(DG_ENOTSUP, "search state does not fit in shared memory (beam/quantizer too large)");
    int &gr = G.granted[key];
    if ((int)smem > gr) {
      DG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      gr = (int)smem;
    }
    auto &per = G.nb[key];
    const uint32_t okey = smem * 8u + wpb;
    auto n_it = per.find(okey);
    if (n_it == per.end()) {
      int v = 0;
      DG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, 32 * (int)wpb, smem));
      n_it = per.emplace(okey, v).first;
    }
    nb = n_it->second;
  }
  if (nb <= 0) return fail(DG_ENOTSUP, "search kernel cannot be resident on an SM");
  if (a.occ_pct > 0 && a.occ_pct < 100) nb = std::max(1, (int)((nb * a.occ_pct + 99) / 100));
  int grid = nb * sms;
  const int need = (int)((a.nq + wpb - 1) / wpb);
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kernel<<<grid, 32 * wpb, smem, st>>>(a, Ly);
  DG_CUDA(cudaGetLastError());
  if (info) {
    info->grid = grid;
    info->blocks_per_sm = nb;
    info->smem = smem;
  }
  return DG_OK;
}

template <int TRAV, int MET, int LPR>
DgStatus launch_trav(const SearchArgs &a, const WarpLayout &Ly, int lcap, bool filt, cudaStream_t st,
                     LaunchInfo *info) {
  constexpr int F = 8;  // lanes per FP32 row in the rerank gather
  switch (lcap) {
    case 64:
      return filt ? launch_persistent(beam_search_kernel<TRAV, MET, LPR, F, 64, true>, a, Ly, st, info)
                  : launch_persistent(beam_search_kernel<TRAV, MET, LPR, F, 64, false>, a, Ly, st, info);
    case 256:
      return filt ? launch_persistent(beam_search_kernel<TRAV, MET, LPR, F, 256, true>, a, Ly, st, info)
                  : launch_persistent(beam_search_kernel<TRAV, MET, LPR, F, 256, false>, a, Ly, st, info);
    case 1024:
      return filt ? launch_persistent(beam_search_kernel<TRAV, MET, LPR, F, 1024, true>, a, Ly, st, info)
                  : launch_persistent(beam_search_kernel<TRAV, MET, LPR, F, 1024, false>, a, Ly, st, info);
    default:
      return fail(DG_EINVAL, "unsupported working-set capacity");
  }
}

template <int TRAV, int LPR>
DgStatus launch_met(const SearchArgs &a, const WarpLayout &Ly, int met, int lcap, bool filt,
                    cudaStream_t st, LaunchInfo *info) {
  switch (met) {
    case MET_L2: return launch_trav<TRAV, MET_L2, LPR>(a, Ly, lcap, filt, st, info);
    case MET_DOT: return launch_trav<TRAV, MET_DOT, LPR>(a, Ly, lcap, filt, st, info);
    default: return launch_trav<TRAV, MET_COS, LPR>(a, Ly, lcap, filt, st, info);
  }
}

// One entry per traversal kind, defined in its own translation unit.
DgStatus launch_search_f32(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                           bool filt, cudaStream_t st, LaunchInfo *info);
DgStatus launch_search_bf16(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                            bool filt, cudaStream_t st, LaunchInfo *info);
DgStatus launch_search_f16(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                           bool filt, cudaStream_t st, LaunchInfo *info);
DgStatus launch_search_int8(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                            bool filt, cudaStream_t st, LaunchInfo *info);
DgStatus launch_search_pq(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                          bool filt, cudaStream_t st, LaunchInfo *info);
DgStatus launch_search_rabitq(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                              bool filt, cudaStream_t st, LaunchInfo *info);
DgStatus launch_search_fp8(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                           bool filt, cudaStream_t st, LaunchInfo *info);

}  // namespace dg
