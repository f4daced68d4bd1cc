// k_c2c.cu -- launcher of the single-pass complex C2C kernels.
#include "fft_launch.cuh"

namespace ffb {

cudaError_t launch_c2c(const C2cArgs& a, int req_logr, cudaStream_t s, uint64_t* launches) {
  C2cIO io{a};
  const int logm = ilog2i(a.N);
  const int logr = choose_logr(logm, req_logr, false);
  if (logr < 0) return cudaErrorInvalidValue;
  return dispatch(io, logm, logr, a.batch, s, launches);
}

}  // namespace ffb
