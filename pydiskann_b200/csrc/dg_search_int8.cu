// int8-code beam search instantiations (Int8Quantizer, src/sq.rs:121-233).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_int8(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                            bool filt, cudaStream_t st, LaunchInfo *info) {
  if (lpr == 8) return launch_met<TRAV_INT8, 8>(a, Ly, met, lcap, filt, st, info);
  if (lpr == 4) return launch_met<TRAV_INT8, 4>(a, Ly, met, lcap, filt, st, info);
  return launch_met<TRAV_INT8, 2>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
