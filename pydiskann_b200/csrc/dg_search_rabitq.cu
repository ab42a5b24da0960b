// RaBitQ-code beam search instantiations (src/rabitq.rs:191-197 estimator).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_rabitq(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                              bool filt, cudaStream_t st, LaunchInfo *info) {
  (void)lpr;
  if (met != MET_L2) return fail(DG_ENOTSUP, "RaBitQ traversal supports l2 metrics only");
  return launch_trav<TRAV_RABITQ, MET_L2, 1>(a, Ly, lcap, filt, st, info);
}
}  // namespace dg
