// PQ-code beam search instantiations: ADC with a shared-memory FP32 table for
// L2 (src/pq.rs:181-209); for cosine / dot the table holds query-centroid
// inner products, i.e. the metric of the decoded code (src/quantized.rs:28-36).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_pq(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                          bool filt, cudaStream_t st, LaunchInfo *info) {
  (void)lpr;
  return launch_met<TRAV_PQ, 1>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
