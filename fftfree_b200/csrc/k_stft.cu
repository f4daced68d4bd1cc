// k_stft.cu -- launcher of the single-pass real-frame STFT kernels.
#include "fft_launch.cuh"

namespace ffb {

cudaError_t launch_stft(const StftArgs& a, int req_logr, cudaStream_t s, uint64_t* launches) {
  const int logm = (a.N == 1) ? 0 : ilog2i(a.N) - 1;
  const int logr = choose_logr(logm, req_logr, true);
  if (logr < 0) return cudaErrorInvalidValue;
  if (a.mag_only == 4) {
    if (post_mode(a.pf) != 0) return cudaErrorInvalidValue;
    return dispatch(StftIO<6>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  }
  if (a.mag_only == 3) return dispatch(StftIO<5>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  if (a.mag_only == 2) return dispatch(StftIO<4>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  if (a.mag_only) return dispatch(StftIO<3>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  switch (post_mode(a.pf)) {
    case 2: return dispatch(StftIO<2>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
    case 1: return dispatch(StftIO<1>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
    default: return dispatch(StftIO<0>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  }
}

long long stft_loss_parts(long long frames, int N) { return frames * loss_slots(N / 2 > 0 ? N / 2 : 1); }

}  // namespace ffb
