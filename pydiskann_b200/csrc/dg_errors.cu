// dg_errors.cu -- per-thread error text, status helpers, the row padding
// rule and the padded row upload, shared by the search library (libdgann) and the index-construction
// library (libdgbuild).
#include <string>

#include "dg_index.h"

namespace dg {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }
DgStatus fail(DgStatus st, const std::string &msg) {
  g_err = msg;
  return st;
}
DgStatus cuda_fail(cudaError_t e, const char *what) {
  g_err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? DG_ENOMEM : DG_EDEVICE;
}

// Rows are padded to a multiple of 32 dimensions: every 16-byte chunk
// geometry of the gather kernels then divides the row exactly.
uint32_t dpad_of(uint32_t d) { return (d + 31u) & ~31u; }

// Copies n host rows of d floats into device rows of dpad floats (zero padded).
DgStatus upload_rows_f32(const float *host, uint64_t n, uint32_t d, uint32_t dpad, float *dev,
                         cudaStream_t st) {
  if (d == dpad) {
    DG_CUDA(cudaMemcpyAsync(dev, host, n * d * sizeof(float), cudaMemcpyHostToDevice, st));
    return DG_OK;
  }
  DG_CUDA(cudaMemsetAsync(dev, 0, n * dpad * sizeof(float), st));
  DG_CUDA(cudaMemcpy2DAsync(dev, dpad * sizeof(float), host, d * sizeof(float), d * sizeof(float), n,
                            cudaMemcpyHostToDevice, st));
  return DG_OK;
}

}  // namespace dg

extern "C" {
const char *dg_last_error(void) { return dg::g_err.c_str(); }
int32_t dg_version(void) { return DGANN_VERSION; }
}
