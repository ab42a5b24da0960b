// FP32-row beam search instantiations (DiskANN::search_with_dists).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_f32(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                           bool filt, cudaStream_t st, LaunchInfo *info) {
  (void)lpr;  // FP32 rows always use 8 lanes per row (dpad is a multiple of 32)
  return launch_met<TRAV_F32, 8>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
