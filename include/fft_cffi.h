/*
 * fft_cffi.h -- C ABI of libfft_cffi.so, the drop-in boundary of the
 * fftfree batched STFT/FFT path, implemented with CUDA kernels for B200.
 *
 * Every declaration below replaces the reference symbol of the same name and
 * signature (reference file fft_cffi.hpp, or ft_tools_cffi.hpp where noted);
 * the cited line is the reference declaration.  Integer constants keep the
 * reference values.  Ownership and error conventions follow the reference:
 * the caller owns every buffer, no exception crosses the ABI, init returns
 * NULL on failure and execute functions return 0 frames / 0 on failure.
 *
 * Pointers may be host memory (pageable or pinned) or CUDA device memory; the
 * library detects which and moves data accordingly.  Calls block until the
 * results are in the caller's buffers unless fftfree_set_async() was enabled
 * and every buffer of the call is device memory (see fftfree_b200.h).
 */
#ifndef FFTFREE_B200_FFT_CFFI_H
#define FFTFREE_B200_FFT_CFFI_H

#include <stddef.h>

#if defined(_WIN32)
#define FFT_CFFI_API __declspec(dllexport)
#else
#define FFT_CFFI_API __attribute__((visibility("default")))
#endif
#ifndef FFTFREE_API
#define FFTFREE_API FFT_CFFI_API
#endif

/* Kernel constants as the reference exports them (fft_cffi.hpp:62-66,
 * derived from eigfft::KernelKind {CooleyTukey, Stockham, External}).  Note
 * that the execute functions read the context's `kernel` as 1 = Cooley-Tukey,
 * 2 = Stockham, anything else = Cooley-Tukey (fft_cffi.cpp:682-686). */
enum { FFT_KERNEL_COOLEYTUKEY = 0, FFT_KERNEL_STOCKHAM = 1, FFT_KERNEL_EXTERNAL = 2 };
/* fft_cffi.hpp:68-73 (eigfft::ButterflyRadix ordinals) */
enum { FFT_BUTTERFLY_RADIX_2 = 0, FFT_BUTTERFLY_RADIX_4 = 1, FFT_BUTTERFLY_RADIX_8 = 2,
       FFT_BUTTERFLY_RADIX_16 = 3 };
/* fft_cffi.hpp:76-81 */
enum { FFT_TRANSFORM_C2C = 0, FFT_TRANSFORM_R2C = 1, FFT_TRANSFORM_C2R = 2, FFT_TRANSFORM_R2R = 3 };
/* fft_cffi.hpp:292-299 */
enum { FFT_WINDOW_RECT = 0, FFT_WINDOW_HANN = 1, FFT_WINDOW_HAMMING = 2, FFT_WINDOW_BLACKMAN = 3,
       FFT_WINDOW_TUKEY = 4, FFT_WINDOW_KAISER = 5 };
/* fft_cffi.hpp:302-306 */
enum { FFT_WINDOW_NORM_NONE = 0, FFT_WINDOW_NORM_L2 = 1, FFT_WINDOW_NORM_AREA = 2 };
/* fft_cffi.hpp:310-313 */
enum { FFT_COLA_OFF = 0, FFT_COLA_NORMALIZE = 1 };
/* fft_cffi.hpp:316-320 */
enum { FFT_STREAM_FLUSH_NONE = 0, FFT_STREAM_FLUSH_PARTIAL = 1, FFT_STREAM_FLUSH_FINAL = 2 };

#ifdef __cplusplus
extern "C" {
#endif

/* fft_cffi.hpp:31 -- one-shot forward transform of n samples, zero-padded to
 * the next power of two; writes the first n bins. */
FFT_CFFI_API void fft_pcm_to_channels(const float* in_pcm, float* out_real, float* out_imag,
                                      float* out_mag, size_t n, int threads);

/* fft_cffi.hpp:90 */
FFT_CFFI_API void* fft_init(size_t n, int threads, int lanes, int inverse, int kernel, int radix,
                            const int* radix_pattern, size_t radix_pattern_len, int pad_mode);

/* fft_cffi.hpp:96 */
FFT_CFFI_API void* fft_init_ex(size_t n, int threads, int lanes, int inverse, int kernel, int radix,
                               const int* radix_pattern, size_t radix_pattern_len, int pad_mode,
                               int window, int hop);

/* fft_cffi.hpp:99-118 */
FFT_CFFI_API void* fft_init_full(size_t n, int threads, int lanes, int inverse, int kernel,
                                 int radix, const int* radix_pattern, size_t radix_pattern_len,
                                 int pad_mode, int window, int hop, int transform,
                                 int reduce_magnitude, int store_polar, int half_spectrum,
                                 int allow_outer_parallel, int allow_inner_parallel,
                                 int inner_threads, int save_crash_logs, int silent_crash_reports);

/* fft_cffi.hpp:121-150 */
FFT_CFFI_API void* fft_init_full_v2(size_t n, int threads, int lanes, int inverse, int kernel,
                                    int radix, const int* radix_pattern, size_t radix_pattern_len,
                                    int pad_mode, int window, int hop, int transform,
                                    int reduce_magnitude, int store_polar, int half_spectrum,
                                    int allow_outer_parallel, int allow_inner_parallel,
                                    int inner_threads, int save_crash_logs,
                                    int silent_crash_reports, int apply_windows, int apply_ola,
                                    int analysis_window_kind, float analysis_param1,
                                    float analysis_param2, int synthesis_window_kind,
                                    float synthesis_param1, float synthesis_param2,
                                    int window_norm_policy, int cola_mode);

/* fft_cffi.hpp:153-158 */
FFT_CFFI_API int fft_execute(void* handle, const float* in_pcm, float* out_real, float* out_imag,
                             float* out_mag, size_t n);

/* fft_cffi.hpp:168-176 -- the batched STFT hot path. */
FFT_CFFI_API size_t fft_execute_batched(void* handle, const float* pcm, size_t pcm_len,
                                        float* out_real, float* out_imag, float* out_mag,
                                        int pad_mode, int enable_backup, size_t max_frames);

/* fft_cffi.hpp:180-186 */
FFT_CFFI_API size_t fft_stft_execute(void* handle, const float* pcm, size_t pcm_len,
                                     float* out_real, float* out_imag, float* out_mag,
                                     size_t max_frames);

/* fft_cffi.hpp:193-211 -- streaming helpers */
FFT_CFFI_API void fft_stream_reset(void* handle);
FFT_CFFI_API size_t fft_stream_push_pcm(void* handle, const float* pcm, size_t samples,
                                        float* out_real, float* out_imag, float* out_mag,
                                        size_t max_frames, int flush_mode);
FFT_CFFI_API size_t fft_stream_pending_frames(void* handle);
FFT_CFFI_API size_t fft_stream_backlog_samples(void* handle);
FFT_CFFI_API size_t fft_stream_push_spectrum(void* handle, const float* in_real,
                                             const float* in_imag, size_t frames, float* out_pcm,
                                             size_t max_samples, int flush_mode);
FFT_CFFI_API size_t fft_stream_pending_pcm(void* handle);

/* fft_cffi.hpp:213-223 */
FFT_CFFI_API int fft_griffin_lim(void* ctx_forward, void* ctx_inverse, const float* in_mag,
                                 size_t frames, int hop, int half_spectrum, int iterations,
                                 int pad_mode, unsigned int seed, float* out_real, float* out_imag);

/* fft_cffi.hpp:228-235 -- inverse / complex-input batch (C2R + OLA path). */
FFT_CFFI_API size_t fft_execute_complex_batched(void* handle, const float* in_real,
                                                const float* in_imag, size_t frames,
                                                float* out_pcm, int pad_mode, int enable_backup,
                                                size_t max_frames);

/* fft_cffi.hpp:237-241 */
FFT_CFFI_API size_t fft_ctx_size(void* handle);
FFT_CFFI_API size_t fft_ctx_worker_threads(void* handle);
FFT_CFFI_API size_t fft_ctx_effective_threads(void* handle);

/* fft_cffi.hpp:246-266 -- test-only dropout controls of the recovery path. */
FFT_CFFI_API void fft_set_workerpool_debug_dropout(int pct);
FFT_CFFI_API void fft_set_workerpool_dropout_pattern(int period, int on_len, int phase);
FFT_CFFI_API void fft_set_workerpool_dropout_single(long long index);
FFT_CFFI_API void fft_set_workerpool_dropout_persistent(int on);
FFT_CFFI_API void fft_clear_workerpool_dropout_history(void);

/* fft_cffi.hpp:270-277 -- phase inference */
FFT_CFFI_API void* phase_init(int N, int hop, int half_spectrum, int mode, int iterations);
FFT_CFFI_API size_t phase_infer_execute(void* handle, const float* in_mag, size_t frames,
                                        float* out_real, float* out_imag);
FFT_CFFI_API void phase_free(void* handle);

/* fft_cffi.hpp:280 */
FFT_CFFI_API void fft_free(void* handle);

/* fft_cffi.hpp:286-287 */
typedef void (*fft_restore_observer_t)(size_t start, size_t end);
FFT_CFFI_API void fft_register_restore_observer(fft_restore_observer_t cb);

/* fft_cffi.hpp:329-345 */
FFT_CFFI_API int fft_config_window(void* handle, int analysis_kind, int synthesis_kind,
                                   float param1, float param2, int norm_policy, int cola_mode);
FFT_CFFI_API int fft_config_window_custom(void* handle, const float* analysis_window,
                                          size_t analysis_len, const float* synthesis_window,
                                          size_t synthesis_len, int norm_policy, int cola_mode);

#ifdef __cplusplus
}
#endif

#endif
