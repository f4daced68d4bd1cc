// kernels.h -- host-side launchers of the sm_100a kernels (C++ linkage,
// internal to libfft_cffi.so).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace ffb {

// Post-transform hook flags (reference eigen_fft.hpp:2535-2596).
struct PostFlags {
  int r2c_half;    // R2C && half_spectrum: DC/Nyquist imag <- 0, bins > N/2 <- 0
  int polar;       // store_polar: (|v|, arg v)
  int reduce;      // reduce_magnitude: (|v|, 0)
  int clear_imag;  // C2R without polar/reduce: imag <- 0
};

// Real frames -> spectrum (fft_execute_batched, fft_execute, fft_pcm_to_channels).
struct StftArgs {
  const float* pcm;
  long long pcm_len;
  long long frames;
  int N, W, H;
  const float* win;  // device, length >= W, or nullptr
  int mirror;        // Cooley-Tukey + C2R + half: x[n] = x[N-n] for n > N/2
  int inverse;
  PostFlags pf;
  int out_bins;
  long long out_stride;
  int mag_from_real;  // out_mag = re when store_polar (fft_cffi.cpp:822)
  float* out_re;   // unused (may be null) with mag_only
  float* out_im;   // unused (may be null) with mag_only
  float* out_mag;
  // Several independent signals: frames [s*sig_frames, (s+1)*sig_frames)
  // read signal s at pcm + s*sig_stride, each `pcm_len` samples long.
  // sig_frames == 0: one signal.
  long long sig_frames;
  long long sig_stride;
  // forward R2C half spectrum, bins 0..N/2: 1 = only |X| (out_mag),
  // 2 = |X| (out_mag) and the unit phasor X / |X| (out_phasor, 0 where |X| = 0),
  // 3 = the residual |X| - target (out_mag), the phasor, and per-warp sums of
  // the squared residuals (loss_part); 4 = the Griffin-Lim projection
  // target e^{i arg X} into (out_re, out_im), no magnitude array (any
  // spectrum layout; post flags without polar or reduce)
  int mag_only;
  float2* out_phasor;
  const float* target;  // mag_only 3 and 4: same layout as the outputs
  float* loss_part;     // mag_only 3: stft_loss_parts(frames, N) floats
};
// Partial sums of the squared residual an L2-loss launch writes.
long long stft_loss_parts(long long frames, int N);

// Gradient of the magnitude STFT (forward R2C half spectrum, |X| per bin)
// with respect to the signals: each frame's spectrum from the saved unit
// phasor or recomputed from the signal, the magnitude chain rule, the
// adjoint transform and the windowed overlap-add adjoint of framing.
struct MagGradArgs {
  const float* pcm;       // signals x sig_stride, each pcm_len samples
  long long signals;
  long long pcm_len;
  long long sig_stride;
  long long frames;       // frames per signal
  int N, W, H;
  const float* win;       // device, length >= W, or nullptr
  const float* grad_mag;  // (signals * frames) x (N/2 + 1)
  const float2* phasor;   // saved X / |X|, same layout (0 at |X| = 0); nullptr: recompute from pcm
  float* grad_pcm;        // signals x sig_stride; every sample < pcm_len written
  int span;               // general form: samples of one signal owned by one block
  int run;                // sliding form: frames of one signal per thread group (0: general form only,
                          // < 0: chosen by the launcher)
  // the gradient is scaled by factor (times *scale when not null, a device
  // scalar: the upstream gradient of a loss, read without a host sync)
  float factor;
  const float* scale;
};

// Complex columns in/out with the plan hooks (C++ fft_inplace_batched).
struct C2cArgs {
  const float2* in;
  float2* out;
  long long batch;
  int N;
  int pre;       // 0 none, 1 R2C imag clear, 2 C2R half mirror (+polar)
  int polar_in;  // polar conversion in pre == 2
  int inverse;
  PostFlags pf;
};

// Planar complex frames -> real frames (fft_execute_complex_batched).
struct CplxBatchArgs {
  const float* in_re;
  const float* in_im;
  long long frames;
  int N, bins;
  int c2r_half;  // Hermitian rebuild of fft_cffi.cpp:1072-1093
  int ct_pre;    // Cooley-Tukey pre-hook: 0 none, 1 R2C imag clear, 2 C2R half
  int polar_in;
  int inverse;
  PostFlags pf;
  const float* synth;  // device window or nullptr
  float* out;          // frames x N
};

struct OlaArgs {
  const float* frames_buf;  // frames x N
  long long frames;
  int N, H;
  int cola;
  const float* weight;  // device, N entries (analysis*synthesis) or nullptr (=1)
  float* out;           // `len` samples
  long long len;        // samples written; 0: frames * N
};

// Twiddle pyramid (levels 0..max_log) on the current device.
const float2* twiddle_pyramid(int max_log, cudaStream_t stream);
// Per-pass twiddle tables of the single-pass engine on the current device.
const float2* twiddle_pass_tables(cudaStream_t stream);

// Pick the single-pass radix (log2) for a transform of 2^logm points;
// `requested_log` (2..4) is honoured when valid, otherwise the tuned
// default for complex (`real_path` false) or real-input paths applies.
// Returns -1 if the size needs the multi-pass path.
int choose_logr(int logm, int requested_log, bool real_path);
int max_single_pass_log();

// Launchers return cudaSuccess or the launch error.  `req_logr` is the
// context's requested pass radix (log2, -1 = default).  `launches` is
// incremented by the number of kernels enqueued.
cudaError_t launch_stft(const StftArgs& a, int logr, cudaStream_t s, uint64_t* launches);
cudaError_t launch_c2c(const C2cArgs& a, int logr, cudaStream_t s, uint64_t* launches);

// Second axis of a 2-D transform: C2C lines whose elements are `rows`
// complex values apart in column-major rows x c.N matrices; line l is row
// (l % rows) of matrix (l / rows), c.batch lines in all.  Single pass, c.N up
// to 2^max_strided_log().  In place (c.in == c.out) is allowed.
struct StridedLinesArgs {
  C2cArgs c;
  long long rows;
  // TMA route: blocks whose bounded wait for their input boxes gave up add 1
  // here (the caller zeroes it before the launch and fails the call when it
  // is non-zero); NULL routes every line through the LSU kernel.
  unsigned* timeouts = nullptr;
};
int max_strided_log();
cudaError_t launch_c2c_strided(const StridedLinesArgs& a, int logr, cudaStream_t s, uint64_t* launches);
// Column-major rows x cols -> cols x rows, `batch` matrices back to back.
cudaError_t launch_transpose(const float2* in, float2* out, long long rows, long long cols, long long batch,
                             cudaStream_t s, uint64_t* launches);
cudaError_t launch_cplx_batch(const CplxBatchArgs& a, int logr, cudaStream_t s, uint64_t* launches);
cudaError_t launch_ola(const OlaArgs& a, cudaStream_t s, uint64_t* launches);
// 256-point C2C transforms (no hooks) on the tcgen05 tensor cores in split
// FP16 (k_tc05.cu), chosen when FFTFREE_TC16=2; the count of blocks whose
// bounded wait on an MMA commit gave up (their outputs are left unwritten).
bool tc05_requested();
cudaError_t launch_c2c256_tc05(const C2cArgs& a, cudaStream_t s, uint64_t* launches);
unsigned tc05_timeouts();

// Griffin-Lim initial spectra: re = mag * cs.x, im = mag * cs.y (cs: the
// cosines and sines of the initial phases).
cudaError_t launch_gl_init(const float* mag, const float2* cs, float* re, float* im, long long n, cudaStream_t s);
// Griffin-Lim projection: re + i im = mag e^{i atan2(ti, tr)} (half spectrum:
// DC and, for even N, Nyquist imaginary parts cleared).
cudaError_t launch_gl_project(const float* mag, const float* tr, const float* ti, float* re, float* im,
                              long long nbins, int bins, int half, int even_n, cudaStream_t s);
// Streaming ISTFT step (fft_cffi.cpp:1597-1742): F inverse frames of N
// samples overlap-added at spacing E = min(hop, N) onto the carried
// accumulator; samples 0 .. count-1 of the sum leave (divided by the summed
// COLA weights when `use_norm` and that sum exceeds 1e-12 in magnitude),
// samples count .. count+N-1 become the next carry (`keep_carry`; else the
// carry is cleared).  Sums run carry first, then frames in order, as the
// reference's frame-by-frame accumulation does.
struct StreamOlaArgs {
  const float* frames;     // F x N
  long long F;
  int N, E;
  const float* carry;      // N
  const float* carry_nrm;  // N (use_norm)
  const float* weight;     // N or nullptr (1)
  int use_norm;
  long long count;
  float* out;              // count samples
  int keep_carry;
  float* new_carry;        // N
  float* new_nrm;          // N (use_norm)
};
cudaError_t launch_stream_ola(const StreamOlaArgs& a, cudaStream_t s);
// Minimum-phase reconstruction (phase inference mode 1): the log-amplitude
// spectrum of every frame (half spectra mirrored), the causal fold of the
// real cepstrum, and exp of the complex log spectrum into planar re / im.
cudaError_t launch_minphase_log(const float* mag, float2* spec, long long frames, int N, int bins, int half,
                                cudaStream_t s);
cudaError_t launch_minphase_fold(float2* cep, long long frames, int N, cudaStream_t s);
cudaError_t launch_minphase_exp(const float2* lg, float* re, float* im, long long frames, int N, int bins,
                                cudaStream_t s);
// Largest N (log2) of the magnitude-gradient kernel; 0 for unsupported.
int max_mag_grad_log();
cudaError_t launch_stft_mag_grad(const MagGradArgs& a, int logr, cudaStream_t s, uint64_t* launches);

// Ragged batch: one persistent launch over items of different sizes (R2C,
// half spectrum, one full frame per item).  tiles[i] = {first item, items,
// log2 complex points, pass radix (log2; 0 for the three-phase sizes)};
// items are listed in tile order, with their signal and output offsets.
// One item of a ragged batch: a real signal of pcm_len samples framed as
// fft_execute_batched frames it with pad_mode 1 (fft_cffi.cpp:710-791:
// frame f covers f*H .. f*H + W, zero-padded to N), its frames' half
// spectra (N/2 + 1 bins each, frame-major) from out_off on.
struct RaggedItem {
  long long pcm_off;  // first sample of the signal in RaggedArgs::pcm
  long long pcm_len;  // samples of the signal
  long long out_off;  // first bin of its first frame in the outputs
  int W, H;           // frame length (<= N) and hop
  int win_off;        // analysis window taps at windows + win_off, -1 for none
  int pad_;
};
struct RaggedArgs {
  const float* pcm;
  float* out_re;
  float* out_im;
  float* out_mag;
  const RaggedItem* items;
  const int2* jobs;     // (item, frame) per frame, tiles' jobs contiguous
  const int4* tiles;    // x first job, y jobs, z log2 of N/2, w pass radix (log2) or 0 (one-block paths)
  int ntiles;
  int* counter;         // tiles handed out; zero before each launch
  float2* scratch;      // ragged_scratch_per_block() bytes per block
  const float* windows; // analysis window taps of every item, concatenated
  PostFlags pf;
};
int ragged_max_log();                 // largest log2 N
int ragged_block_log(int logm);       // sizes one block takes alone: 1, else 0
size_t ragged_scratch_per_block();
int ragged_candidates(int logm, int* lrs);  // pass radices (log2) a size may use
int ragged_grid();                    // persistent blocks for the current device
int ragged_block_threads();           // threads per block of the persistent kernel
cudaError_t launch_ragged(const RaggedArgs& a, int grid, cudaStream_t s, uint64_t* launches);

// Multi-pass (four-step) transforms for 2^14 <= N <= 2^20.  `scratch` holds
// `chunk` transforms of N complex points (four_step_chunk picks the chunk:
// up to 1 GiB of scratch by default).
int max_multi_pass_log();
size_t four_step_chunk(int log_n, long long batch);
cudaError_t launch_four_step_stft(const StftArgs& a, float2* scratch, size_t chunk, cudaStream_t s,
                                  uint64_t* launches);
cudaError_t launch_four_step_c2c(const C2cArgs& a, float2* scratch, size_t chunk, cudaStream_t s,
                                 uint64_t* launches);
cudaError_t launch_four_step_cplx(const CplxBatchArgs& a, float2* scratch, size_t chunk, cudaStream_t s,
                                  uint64_t* launches);

}  // namespace ffb
