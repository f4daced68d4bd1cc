/*
 * fftfree_b200.h -- additive extensions of libfft_cffi.so (B200 build).
 *
 * These entry points have no C-ABI counterpart in the reference; each one
 * names the reference C++ API it exposes.  All keep the reference
 * conventions: plain pointers and sizes, 0 on failure, no exceptions.
 */
#ifndef FFTFREE_B200_EXT_H
#define FFTFREE_B200_EXT_H

#include <stddef.h>
#include "fft_cffi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Complex-in / complex-out batched transform with the context's plan flags
 * (transform mode, hooks, inverse, kernel) -- the reference C++ API
 * eigfft::fft_inplace_batched (eigen_fft.hpp:3170-3175), which the reference
 * C ABI does not expose (its complex entry returns only the real part).
 * `in` and `out` hold `batch` transforms of N interleaved complex floats
 * each (the N x batch column-major matrix of the C++ API); they may alias.
 * Returns 1 on success. */
FFT_CFFI_API int fftfree_execute_c2c(void* handle, const float* in, float* out, size_t batch);

/* 2-D transform of `batch` column-major rows x cols complex matrices --
 * eigfft::fft_inplace_2d (eigen_fft.hpp:3177-3215): the plan of ctx_axis0
 * (N = rows) over every column, then the plan of ctx_axis1 (N = cols) over
 * every row, each with its context's flags (direction, 1/N on inverse,
 * hooks).  `in` / `out` hold batch * rows * cols interleaved complex floats,
 * matrix after matrix; they may alias (the reference works in place).
 * Returns 0 when a context's N does not match its axis (the reference throws
 * std::invalid_argument there), 1 on success.  Runs on ctx_axis0's stream.
 * The row pass moves its lines with TMA where the layout allows; its waits for
 * the copies are bounded, and a block whose wait gives up leaves its lines
 * unwritten and is counted: a synchronous call then returns 0, an
 * asynchronous one (fftfree_set_async on device buffers) makes the next
 * fftfree_execute_2d call on ctx_axis0 return 0. */
FFT_CFFI_API int fftfree_execute_2d(void* ctx_axis0, void* ctx_axis1, const float* in, float* out, size_t rows,
                                    size_t cols, size_t batch);

/* One metadata request: the fields of eigfft::MetadataRequest
 * (eigen_fft.hpp:1496-1501); `buffer` holds `count` interleaved complex
 * floats.  Kinds are eigfft::MetadataKind ordinals (eigen_fft.hpp:1477-1491):
 * 0 Twiddle, 1 LayoutMap, 2 StageSnapshot, 3 StageParams, 4 ButterflyPairs,
 * 5 StageInvariant, 6 TwiddleIndexMap, 7 Omega, 8 StageSnapshotAll,
 * 9 ButterflyPairsAll, 10 TwiddleIndexMapAll. */
typedef struct fftfree_metadata_request {
  int kind;
  float* buffer;
  size_t count;
} fftfree_metadata_request;

/* eigfft::fft_inplace_batched_with_metadata (eigen_fft.hpp:3152-3168): the
 * transform of fftfree_execute_c2c executed as the literal radix-2 stage
 * sequence of the context's kernel (Cooley-Tukey or Stockham), filling the
 * requested metadata.  Returns 0 when a buffer is too small (the reference
 * throws std::invalid_argument there). */
FFT_CFFI_API int fftfree_execute_c2c_meta(void* handle, const float* in, float* out, size_t batch,
                                          const fftfree_metadata_request* requests,
                                          int request_count);

/* Run the context's work on this CUDA stream (a cudaStream_t, used as given:
 * NULL is CUDA's legacy default stream).  A context starts on a non-blocking
 * stream of its own; fftfree_ctx_stream() returns the current one, so a
 * caller can put it back later. */
FFT_CFFI_API void fftfree_set_stream(void* handle, void* cuda_stream);

/* The CUDA stream the context currently runs on. */
FFT_CFFI_API void* fftfree_ctx_stream(void* handle);

/* When on, a call whose buffers are all device memory returns once its work
 * is enqueued on the context stream instead of waiting for it. */
FFT_CFFI_API void fftfree_set_async(void* handle, int on);

/* Number of kernels this context has launched so far. */
FFT_CFFI_API unsigned long long fftfree_ctx_launch_count(void* handle);

/* Radix schedule (per pass) that the context's plan executes for its main
 * transform; returns the number of passes written (at most max_passes). */
FFT_CFFI_API int fftfree_ctx_schedule(void* handle, int* radices, int max_passes);

/* The context's executor code after the FFTFREE_DEFAULT_KERNEL override of
 * fft_init / fft_init_ex (fft_cffi.cpp:126-159, 553-558): 0 auto
 * (Cooley-Tukey), 1 Cooley-Tukey, 2 Stockham; -1 for a NULL handle. */
FFT_CFFI_API int fftfree_ctx_kernel(void* handle);

/* Frames fft_execute_batched would produce for pcm_len samples with this
 * pad_mode and max_frames (the rule of fft_cffi.cpp:710-750), and the
 * context's effective frame length W and hop H (window / hop, 0 -> N / W):
 * what a caller needs to split one signal's frames over several GPUs. */
FFT_CFFI_API size_t fftfree_frame_count(void* handle, size_t pcm_len, int pad_mode, size_t max_frames);
FFT_CFFI_API int fftfree_ctx_frame_shape(void* handle, int* window, int* hop);

/* 1 when a CUDA device is usable by this library, else 0. */
FFT_CFFI_API int fftfree_device_available(void);

/* No counterpart in the reference.  fft_execute_complex_batched (fast path,
 * with the context's windows and overlap-add) for callers that cannot
 * allocate GPU memory while they run -- a real-time audio thread, for which
 * cudaMalloc / cudaFree may block and synchronise the device, or a process
 * whose GPU memory is all reserved up front by another allocator.  The call
 * allocates nothing: all three buffers must be device memory (host buffers
 * are rejected, they would need staging), and the per-frame samples that the
 * overlap-add sums are kept in a fixed 16 MiB array compiled into the
 * library, which every GPU that loads the library holds until exit.  Limits:
 * frames * N <= 4,194,304 when the context applies overlap-add, and N up to
 * 8192 points (16384 for a half-spectrum C2R context), the sizes one pass
 * covers; other calls are rejected with a message on stderr and return 0.
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture.  With
 * CUDA's lazy module loading (the default), the first launch of each kernel
 * loads its code, which may itself take device memory: make one call with
 * each context (this entry point or fft_execute_complex_batched) before the
 * time-critical path.  All calls share the array and it keeps the last
 * call's contents (every sample is rewritten before it is read): calls that
 * overlap on the GPU (other streams, other contexts) race on it.
 * Returns the frames produced, 0 on failure. */
FFT_CFFI_API size_t fftfree_execute_complex_batched_noalloc(void* handle, const float* in_real,
                                                           const float* in_imag, size_t frames,
                                                           float* out_pcm, size_t max_frames);

/* Differentiable STFT magnitude, the forward and adjoint kernels behind a
 * torch.autograd.Function.  No C counterpart in the reference; it replaces
 * the forward-STFT approximation of the adjoint that train_mipmap_weights.py
 * (lines 395-415) uses for its spectral losses.  The context must be a
 * forward R2C half-spectrum context (fft_init_full / fft_init_full_v2 with
 * transform=1, half_spectrum=1) with N <= 16384; N, window length W, hop H,
 * the pad rule of fft_execute_batched (fft_cffi.cpp:710-750) and the
 * analysis window (apply_windows=1) come from it.
 *
 * fftfree_stft_magnitude: |X| of every frame of `signals` signals, each
 * `length` samples at row stride `length`, into out_mag as
 * signals x frames x (N/2 + 1) floats (frames per signal as
 * fft_execute_batched counts them, capped by max_frames when nonzero); the
 * same framing, window and kernels as fft_execute_batched with
 * reduce_magnitude.  Returns the frames per signal, 0 on failure. */
FFT_CFFI_API size_t fftfree_stft_magnitude(void* handle, const float* pcm, size_t signals, size_t length,
                                           float* out_mag, size_t max_frames);

/* Gradient of sum(grad_mag * |X|) with respect to pcm: grad_mag has the
 * layout of fftfree_stft_magnitude's output (all frames of every signal),
 * grad_pcm receives signals x length floats.  The spectrum is recomputed
 * from pcm, not stored; bins with |X| = 0 contribute nothing; samples no
 * frame covers get 0.  Deterministic (no atomics).  Returns the frames per
 * signal, 0 on failure. */
FFT_CFFI_API size_t fftfree_stft_magnitude_backward(void* handle, const float* pcm, size_t signals,
                                                    size_t length, const float* grad_mag, float* grad_pcm);

/* The forward pass that keeps what the gradient needs instead of the
 * signal: |X| into out_mag as fftfree_stft_magnitude does, and the unit
 * phasor X / |X| (0 where |X| = 0) into out_phasor as interleaved
 * (real, imaginary) float pairs, signals x frames x (N/2 + 1) of them.
 * Returns the frames per signal, 0 on failure. */
FFT_CFFI_API size_t fftfree_stft_magnitude_phasor(void* handle, const float* pcm, size_t signals, size_t length,
                                                  float* out_mag, float* out_phasor, size_t max_frames);

/* fftfree_stft_magnitude_backward from the phasor fftfree_stft_magnitude_phasor
 * saved instead of the signal: one inverse transform per frame, no forward
 * transform.  length is the signals' length (it fixes the frames and the last
 * frame's sample count).  Returns the frames per signal, 0 on failure. */
FFT_CFFI_API size_t fftfree_stft_magnitude_backward_phasor(void* handle, const float* phasor, size_t signals,
                                                           size_t length, const float* grad_mag,
                                                           float* grad_pcm);

/* The spectral L2 loss sum((|X| - target)^2) in one pass: |X| - target into
 * out_residual (target and residual with the layout of
 * fftfree_stft_magnitude's output), the unit phasor into out_phasor, and the
 * squared residuals summed per frame into fftfree_stft_l2_partials(handle,
 * signals * frames) partial sums in out_partials (their sum is the loss; a
 * fixed summation order, no atomics).  Its gradient is
 * fftfree_stft_magnitude_backward_phasor_scaled(phasor, grad_mag = residual,
 * scale = the loss's upstream gradient, factor = 2).  Returns the frames per
 * signal, 0 on failure. */
FFT_CFFI_API size_t fftfree_stft_l2_partials(void* handle, size_t frames_total);
FFT_CFFI_API size_t fftfree_stft_magnitude_l2(void* handle, const float* pcm, size_t signals, size_t length,
                                              const float* target, float* out_residual, float* out_phasor,
                                              float* out_partials, size_t max_frames);

/* fftfree_stft_magnitude_backward_phasor with the gradient scaled by factor,
 * times *scale when scale is not NULL (a device pointer to one float, read by
 * the kernel: an upstream gradient that never visits the host). */
FFT_CFFI_API size_t fftfree_stft_magnitude_backward_phasor_scaled(void* handle, const float* phasor,
                                                                  size_t signals, size_t length,
                                                                  const float* grad_mag, float* grad_pcm,
                                                                  const float* scale, float factor);

/* Ragged batches.  No counterpart in the reference, whose callers create
 * one context per transform size and loop over the transforms
 * (fft_init_full + fft_execute_batched per size).  A plan covers `count`
 * real signals of sizes[i] samples each (powers of two, 4 .. 65536), packed
 * back to back; item i gives what fft_execute_batched gives for one frame of
 * it on a context (sizes[i], window = hop = sizes[i], transform = R2C,
 * half_spectrum = 1, the plan's reduce_magnitude / store_polar): planar
 * re / im / mag rows of sizes[i]/2 + 1 bins, packed back to back in item
 * order.  All items run in one persistent kernel launch (captured once in a
 * CUDA graph per set of buffers); the pass radix of each size is chosen by
 * timing the candidates on the plan's own items at plan time, cached in
 * FFTFREE_TUNE_CACHE (default ~/.cache/fftfree_b200/tune.txt) keyed by
 * (size, items of that size, transform); FFTFREE_TUNE=0 keeps the defaults.
 * The plan lives on the device current at creation.  Returns NULL on a bad
 * size or a CUDA failure. */
FFT_CFFI_API void* fftfree_ragged_plan(const size_t* sizes, size_t count, int reduce_magnitude,
                                       int store_polar);
/* The same for ragged mixes of size AND framing: item i is a real signal of
 * lengths[i] samples framed as fft_execute_batched frames it with pad_mode 1
 * on a context (n[i], window[i], hop[i], transform = R2C, half_spectrum = 1,
 * apply_windows with analysis window kind window_kind[i] and parameter
 * window_param[i], norm policy 0) (fft_cffi.cpp:701-824, 163-208): frames of
 * window[i] <= n[i] samples every hop[i] samples, zero-padded to n[i]
 * (powers of two, 4 .. 65536), a lone partial frame when the signal is
 * shorter than one.  Its frames' planar rows of n[i]/2 + 1 bins are packed
 * frame after frame, items in order.  window, hop, window_kind and
 * window_param may be NULL (window = hop = n, rectangular); window[i] or
 * hop[i] of 0 means n[i] (hop: window[i]). */
FFT_CFFI_API void* fftfree_ragged_plan_stft(const size_t* n, const size_t* lengths, const int* window,
                                            const int* hop, const int* window_kind, const float* window_param,
                                            size_t count, int reduce_magnitude, int store_polar);
/* Frames the plan computes for item i (0 for a bad index). */
FFT_CFFI_API size_t fftfree_ragged_frames(void* plan, size_t item);
/* Total input samples / output bins per array of a plan (0 for NULL). */
FFT_CFFI_API size_t fftfree_ragged_samples(void* plan);
FFT_CFFI_API size_t fftfree_ragged_bins(void* plan);
/* The pass radix the plan runs for size n (0: n is absent from the plan's
 * single-pass sizes, or takes the two-half path of 65536 points). */
FFT_CFFI_API int fftfree_ragged_schedule(void* plan, size_t n);
/* Frames of size n per tile that a block of the plan's launch claims at once
 * (one or more block-loads, the tuner's tile size; 1 for the sizes that take
 * a whole block per frame, 0 for a NULL plan or an unsupported n). */
FFT_CFFI_API int fftfree_ragged_tile(void* plan, size_t n);
/* Stream of the plan's launches (NULL: the plan's own stream). */
FFT_CFFI_API void fftfree_ragged_set_stream(void* plan, void* cuda_stream);
/* Runs the plan: host or device buffers (host ones are staged and the call
 * waits; with device buffers it returns once the launch is enqueued).
 * Returns 1, or 0 on failure. */
FFT_CFFI_API int fftfree_ragged_execute(void* plan, const float* pcm, float* out_real, float* out_imag,
                                        float* out_mag);
/* Graph launches this plan has issued (one per execute). */
FFT_CFFI_API unsigned long long fftfree_ragged_launch_count(void* plan);
FFT_CFFI_API void fftfree_ragged_free(void* plan);

/* Test hook of the recovery coordinator (fft_cffi.cpp:954-982): runs the
 * host-side dropout / restore / split decisions for one batch of `frames`
 * frames, invoking the registered restore observer as the recovery path
 * would, and writes 1 into raw_out[f] for each frame left in its restored
 * (untransformed) state.  Needs no GPU.  Returns the number of such frames. */
FFT_CFFI_API size_t fftfree_debug_recovery_plan(size_t frames, char* raw_out);

#ifdef __cplusplus
}
#endif

#endif
