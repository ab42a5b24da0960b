// FP8 (e4m3, per-vector scales) beam search instantiations; q.x on the tensor
// cores with FP32 accumulation.  No counterpart in the reference.
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_fp8(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                           bool filt, cudaStream_t st, LaunchInfo *info) {
  (void)lpr;
  return launch_met<TRAV_FP8, 1>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
