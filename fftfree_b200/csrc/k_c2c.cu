// k_c2c.cu -- launcher of the single-pass complex C2C kernels.
#include "fft_launch.cuh"

namespace ffb {

cudaError_t launch_c2c(const C2cArgs& a, int req_logr, cudaStream_t s, uint64_t* launches) {
  // FFTFREE_TC16=2: plain 256-point transforms on the tcgen05 tensor cores
  // in split FP16 (k_tc05.cu)
  if (a.N == 256 && a.pre == 0 && !(a.pf.r2c_half | a.pf.polar | a.pf.reduce | a.pf.clear_imag) &&
      tc05_requested())
    return launch_c2c256_tc05(a, s, launches);
  C2cIO io{a};
  const int logm = ilog2i(a.N);
  const int logr = choose_logr(logm, req_logr, false);
  if (logr < 0) return cudaErrorInvalidValue;
  return dispatch(io, logm, logr, a.batch, s, launches);
}

}  // namespace ffb
