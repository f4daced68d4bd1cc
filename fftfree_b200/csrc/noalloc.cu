// noalloc.cu -- fftfree_execute_complex_batched_noalloc: the inverse /
// complex-input batch with overlap-add, for callers that must not allocate
// GPU memory while they run.
//
// Who needs it: a real-time audio thread that turns spectra back into PCM
// cannot afford cudaMalloc / cudaFree, which may block for a long time and
// synchronise the whole device, and a process whose GPU memory was handed
// out up front to another allocator may find that a fresh cudaMalloc fails.
// Such callers create the context (which allocates) at set-up time and then
// call this entry point from the time-critical path.
//
// The overlap-add needs every frame's time-domain samples before it can sum
// them; fft_execute_complex_batched keeps those in a device buffer that the
// context grows on demand.  Here they live in a fixed file-scope __device__
// array instead, so the call itself allocates nothing.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/fftfree_b200.h"
#include "context.h"
#include "kernels.h"

namespace ffb {
namespace {

// Largest frames * N the scratch holds: 4,194,304 samples (16 MiB).  Every
// GPU that loads this library keeps this array until the process exits.
constexpr size_t kNoAllocMaxSamples = (size_t)1 << 22;

__device__ __align__(256) float g_noalloc_frames[kNoAllocMaxSamples];

// In host code `g_noalloc_frames` names a host-side stand-in, not device
// memory: the kernels get the device address looked up here, once per
// device, with that device current.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_scratch[kMaxDevices] = {};

float* scratch_address(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev]) {
    float* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_frames);
    if (e != cudaSuccess) {
      std::fprintf(stderr, "[fftfree_b200] fftfree_execute_complex_batched_noalloc: "
                           "cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return nullptr;
    }
    g_scratch[dev] = p;
  }
  return g_scratch[dev];
}

bool on_device(const void* p) {
  cudaPointerAttributes at;
  if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" FFT_CFFI_API size_t fftfree_execute_complex_batched_noalloc(void* handle, const float* in_real,
                                                                       const float* in_imag, size_t frames,
                                                                       float* out_pcm, size_t max_frames) {
  FftContext* c = as_ctx(handle);
  if (!c || !in_real || !in_imag || !out_pcm || frames == 0 || c->N <= 0) return 0;
  if (max_frames != 0 && frames > max_frames) frames = max_frames;
  const int N = c->N;
  const size_t samples = frames * (size_t)N;
  if (c->apply_ola && samples > kNoAllocMaxSamples) {
    std::fprintf(stderr, "[fftfree_b200] fftfree_execute_complex_batched_noalloc: frames * N = %zu exceeds "
                         "the fixed scratch of %zu samples\n", samples, kNoAllocMaxSamples);
    return 0;
  }
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != c->device) cudaSetDevice(c->device);
  size_t result = 0;
  do {
    if (!on_device(in_real) || !on_device(in_imag) || !on_device(out_pcm)) {
      std::fprintf(stderr, "[fftfree_b200] fftfree_execute_complex_batched_noalloc: buffers must be device "
                           "memory (host buffers would need staging allocations)\n");
      break;
    }
    // one-pass sizes only (the multi-pass kernels need a scratch chunk): the
    // half-spectrum C2R path runs an N/2-point transform, the others N points
    const bool c2r_half_path = c->half_spectrum && c->eff_transform() == 2 && N >= 4;
    if (ilog2i(N) - (c2r_half_path ? 1 : 0) > max_single_pass_log()) {
      std::fprintf(stderr, "[fftfree_b200] fftfree_execute_complex_batched_noalloc: N=%d not supported "
                           "(one-pass sizes only)\n", N);
      break;
    }
    float* frames_buf = out_pcm;
    if (c->apply_ola) {
      frames_buf = scratch_address(c->device);
      if (!frames_buf) break;
    }
    // Same arguments as fft_execute_complex_batched (fft_cffi.cpp:1042-1162).
    CplxBatchArgs a{};
    a.in_re = in_real;
    a.in_im = in_imag;
    a.frames = (long long)frames;
    a.N = N;
    a.bins = c->bins();
    const int m = c->eff_transform();
    a.c2r_half = (c->half_spectrum && m == 2) ? 1 : 0;
    a.ct_pre = c->stockham() ? 0 : (m == 1 ? 1 : ((m == 2 && c->half_spectrum) ? 2 : 0));
    a.polar_in = c->store_polar ? 1 : 0;
    a.inverse = c->inverse ? 1 : 0;
    a.pf = c->post_flags();
    a.synth = c->windows_enabled ? static_cast<const float*>(c->d_synthesis.p) : nullptr;
    a.out = frames_buf;
    // The transform writes every one of the frames * N scratch samples before
    // the overlap-add reads them, so nothing has to be cleared between calls.
    if (launch_cplx_batch(a, c->logr_req, c->stream, &c->launches) != cudaSuccess) break;
    if (c->apply_ola) {
      OlaArgs o{};
      o.frames_buf = frames_buf;
      o.frames = (long long)frames;
      o.N = N;
      o.H = (c->hop > 0) ? c->hop : ((c->window > 0) ? c->window : N);
      o.cola = (c->cola_mode == FFT_COLA_NORMALIZE) ? 1 : 0;
      o.weight = c->windows_enabled ? static_cast<const float*>(c->d_weight.p) : nullptr;
      o.out = out_pcm;
      if (launch_ola(o, c->stream, &c->launches) != cudaSuccess) break;
    }
    if (cudaGetLastError() != cudaSuccess) break;
    if (!c->async && cudaStreamSynchronize(c->stream) != cudaSuccess) break;
    result = frames;
  } while (false);
  if (prev >= 0 && prev != c->device) cudaSetDevice(prev);
  return result;
}
