// F16-code beam search instantiations (F16Quantizer, src/sq.rs:36-108).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_f16(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                           bool filt, cudaStream_t st, LaunchInfo *info) {
  if (lpr == 8) return launch_met<TRAV_F16, 8>(a, Ly, met, lcap, filt, st, info);
  return launch_met<TRAV_F16, 4>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
