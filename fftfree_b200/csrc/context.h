// context.h -- the FftContext behind the opaque handle of libfft_cffi.so.
//
// Mirrors the fields of the reference context (fft_cffi.cpp:40-82) and adds
// the device state that replaces the reference's PlanCache + WorkerPool: one
// CUDA stream, device-resident windows and grow-only staging buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "kernels.h"

namespace ffb {

// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  void* get(size_t bytes);
  void release();
  ~DevBuf() { release(); }
};

struct FftContext {
  uint32_t magic = 0x46465442u;  // "FFTB"
  // --- reference fields ---
  int N = 0;
  bool inverse = false;
  int kernel = 0;  // 0 = auto (Cooley-Tukey), 1 = Cooley-Tukey, 2 = Stockham
  int radix = 0;
  int pad_mode = 0;
  std::vector<int> radix_pattern;
  int window = 0;
  int hop = 0;
  int transform = 0;
  int reduce_magnitude = 0;
  int store_polar = 0;
  int half_spectrum = 0;
  int allow_outer_parallel = 1;
  int allow_inner_parallel = 0;
  int inner_threads = 0;
  int threads = 1;  // PlanRuntimeConfig::threads as the reference stores it
  int lanes = 1;
  bool has_pool = false;  // the reference creates a WorkerPool here
  int analysis_win_kind = 0, synthesis_win_kind = 0;
  float win_param1 = 0.f, win_param2 = 0.f;
  int win_norm_policy = 0, cola_mode = 0;
  std::vector<float> analysis_win, synthesis_win;
  bool windows_enabled = false;
  int apply_ola = 0;
  // streaming state (fft_cffi.cpp:72-78), resident on the device:
  //  * the pushed samples not yet consumed are [s_off, s_end) of d_stream
  //    (d_stream2: the target of a compaction when it fills up);
  //  * the inverse side's overlap-add carry (acc_len = 0 or N) and COLA norm
  //    (nrm_len = 0 or N), double-buffered;
  //  * emitted samples waiting for the caller are [q_off, q_end) of d_queue.
  DevBuf d_stream, d_stream2;
  size_t s_off = 0, s_end = 0;
  DevBuf d_acc, d_acc2, d_nrm, d_nrm2, d_ifr, d_sweight;
  size_t acc_len = 0, nrm_len = 0;
  int sweight_n = 0;
  DevBuf d_queue, d_queue2;
  size_t q_off = 0, q_end = 0;
  DevBuf d_sre, d_sim, d_smg;  // push_pcm outputs the caller leaves NULL
  // Griffin-Lim working set, kept on the forward context between calls:
  // magnitudes and spectra, the inverse's frames, the overlap-added signal,
  // the unfused forward outputs; the generator's state words and the
  // initial phasors in pinned host memory
  DevBuf d_gl_spec, d_gl_frames, d_gl_ola, d_gl_tmp;
  std::vector<uint32_t> h_gl_state;
  float2* h_gl_cs = nullptr;
  size_t h_gl_cs_cap = 0;

  // --- device state ---
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool async = false;
  int logr_req = -1;  // requested pass radix (log2), -1 = autotuned default
  DevBuf d_analysis, d_synthesis, d_weight;
  bool windows_uploaded = false;
  DevBuf d_in0, d_in1, d_out0, d_out1, d_out2, d_frames;
  DevBuf d_meta_tw;  // reference float twiddle table for the metadata path
  DevBuf d_scratch;  // multi-pass intermediate chunk
  DevBuf d_t2d;      // transposed matrices of a 2-D transform with long rows
  // 2-D row pass through TMA: the device count of blocks whose bounded wait
  // gave up (cumulative until a call reports it) and its pinned host copy,
  // refreshed by every such call when its stream reaches the copy
  DevBuf d_tma_timeouts;
  unsigned* h_tma_timeouts = nullptr;
  // host-buffer pipeline (abi.cpp): upload / download streams and events
  cudaStream_t up_stream = nullptr, down_stream = nullptr;
  std::vector<cudaEvent_t> pipe_events;
  uint64_t launches = 0;
  std::recursive_mutex mu;

  int eff_transform() const { return (transform >= 0 && transform <= 3) ? transform : 0; }
  bool stockham() const { return kernel == 2; }
  int bins() const { return half_spectrum ? N / 2 + 1 : N; }
  PostFlags post_flags() const;
};

FftContext* as_ctx(void* h);

// The W taps of an analysis / synthesis window as the contexts build them
// (fft_cffi.cpp:163-208: kind, parameter p1, normalisation policy).
std::vector<float> window_taps(int kind, int W, float p1, float p2, int norm_policy);

// One Griffin-Lim iteration's transforms on device buffers, enqueued on the
// context's stream with no host synchronisation (they throw on CUDA errors):
// the inverse batch of (re, im) into frame_pcm, and the forward STFT of pcm
// whose spectra are projected onto the magnitudes mag into (re, im) -- by
// the STFT's own epilogue where the plan allows, else through (tr, ti, tm)
// and a projection kernel.  Each returns the frames it produced, 0 if none.
size_t gl_inverse_enqueue(FftContext* c, const float* re, const float* im, size_t frames, float* frame_pcm);
size_t gl_forward_project_enqueue(FftContext* c, const float* pcm, size_t pcm_len, int pad_mode,
                                  size_t max_frames, const float* mag, float* re, float* im, int bins,
                                  bool half, bool even_n, float* tr, float* ti, float* tm);

}  // namespace ffb
