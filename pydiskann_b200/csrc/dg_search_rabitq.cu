// RaBitQ-code beam search instantiations: the estimator for L2
// (src/rabitq.rs:191-197); for cosine / dot the decoded code's inner product
// with the query, evaluated in the rotated space (src/rabitq.rs:224-238,
// src/quantized.rs:28-36).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_rabitq(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                              bool filt, cudaStream_t st, LaunchInfo *info) {
  (void)lpr;
  return launch_met<TRAV_RABITQ, 1>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
