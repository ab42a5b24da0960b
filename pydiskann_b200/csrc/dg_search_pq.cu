// PQ-code beam search instantiations (ADC with a shared-memory FP32 table).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_pq(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                          bool filt, cudaStream_t st, LaunchInfo *info) {
  (void)lpr;
  if (met != MET_L2) return fail(DG_ENOTSUP, "PQ traversal supports l2 metrics only");
  return launch_trav<TRAV_PQ, MET_L2, 1>(a, Ly, lcap, filt, st, info);
}
}  // namespace dg
