// BF16-row beam search instantiations (FP32 accumulate, optional FP32 rerank).
#include "dg_launch.cuh"
namespace dg {
DgStatus launch_search_bf16(const SearchArgs &a, const WarpLayout &Ly, int met, int lpr, int lcap,
                            bool filt, cudaStream_t st, LaunchInfo *info) {
  if (lpr == 8) return launch_met<TRAV_BF16, 8>(a, Ly, met, lcap, filt, st, info);
  return launch_met<TRAV_BF16, 4>(a, Ly, met, lcap, filt, st, info);
}
}  // namespace dg
