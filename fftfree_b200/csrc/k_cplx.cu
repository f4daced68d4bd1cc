// k_cplx.cu -- launcher of the single-pass complex / inverse batch kernels.
#include "fft_launch.cuh"

namespace ffb {

cudaError_t launch_cplx_batch(const CplxBatchArgs& a, int req_logr, cudaStream_t s, uint64_t* launches) {
  const int lg = ilog2i(a.N);
  if (a.c2r_half && a.N >= 4) {
    C2rHalfIO io{a, lg};
    const int logr = choose_logr(lg - 1, req_logr, true);
    if (logr < 0) return cudaErrorInvalidValue;
    return dispatch(io, lg - 1, logr, a.frames, s, launches);
  }
  CplxBatchIO io{a};
  const int logr = choose_logr(lg, req_logr, false);
  if (logr < 0) return cudaErrorInvalidValue;
  return dispatch(io, lg, logr, a.frames, s, launches);
}

}  // namespace ffb
