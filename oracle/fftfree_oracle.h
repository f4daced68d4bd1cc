/*
 * fftfree_oracle.h -- CPU restatement of the fftfree batched STFT/FFT path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in fftfree_b200/: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it.  The product library never links
 * or calls it.
 *
 * It restates, in plain C and float32 arithmetic, the algorithm of the
 * reference (sangderenard/fftfree) for the hot path:
 *   - Plan twiddles / bit reversal          eigen_fft.hpp:2229-2253
 *   - Cooley-Tukey executor                 eigen_fft.hpp:2655-3100
 *   - Stockham executor                     eigen_fft.hpp:3227-3623
 *   - pre/post transform hooks              eigen_fft.hpp:2484-2596
 *   - metadata writers                      eigen_fft.hpp:1477-1888
 *   - STFT framing + output copy            fft_cffi.cpp:701-1034
 *   - complex/inverse batch + OLA/COLA      fft_cffi.cpp:1042-1340
 *   - window construction / normalisation   fft_cffi.cpp:163-208
 *   - context init rules                    fft_cffi.cpp:535-658, 1792-1978
 *
 * The reference needs Eigen 3.4.0 (fetched by CMake, not vendored, absent
 * here), so it is not built; this restatement is pinned instead against the
 * known-answer cases of the reference's own tests (tests/golden/).
 */
#ifndef FFTFREE_ORACLE_H
#define FFTFREE_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of the reference FftContext fields that affect results
 * (fft_cffi.cpp:40-82).  Windows are length N (first W taps from the window
 * builder, the rest 1.0; fft_cffi.cpp:1893-1906). */
typedef struct oracle_cfg {
  int N;
  int inverse;
  int kernel;        /* 0 = auto (Cooley-Tukey), 1 = Cooley-Tukey, 2 = Stockham */
  int transform;     /* 0 C2C, 1 R2C, 2 C2R, 3 R2R (others -> C2C) */
  int reduce_magnitude;
  int store_polar;
  int half_spectrum;
  int window;        /* W (0 -> N) */
  int hop;           /* H (0 -> W) */
  int pad_mode;      /* context pad mode */
  int windows_enabled;
  int apply_ola;
  int cola_mode;
  const float* analysis_win;   /* length N or NULL */
  const float* synthesis_win;  /* length N or NULL */
} oracle_cfg;

/* Metadata request, same meaning as eigfft::MetadataRequest
 * (eigen_fft.hpp:1496-1501); buf holds `count` interleaved complex floats. */
typedef struct oracle_meta_req {
  int kind;
  float* buf;
  size_t count;
} oracle_meta_req;

enum {
  ORACLE_META_TWIDDLE = 0,
  ORACLE_META_LAYOUT_MAP = 1,
  ORACLE_META_STAGE_SNAPSHOT = 2,
  ORACLE_META_STAGE_PARAMS = 3,
  ORACLE_META_BUTTERFLY_PAIRS = 4,
  ORACLE_META_STAGE_INVARIANT = 5,
  ORACLE_META_TWIDDLE_INDEX_MAP = 6,
  ORACLE_META_OMEGA = 7,
  ORACLE_META_STAGE_SNAPSHOT_ALL = 8,
  ORACLE_META_BUTTERFLY_PAIRS_ALL = 9,
  ORACLE_META_TWIDDLE_INDEX_MAP_ALL = 10
};

/* Plan twiddle table W[k], k < max(1, N/2), float angle arithmetic as in the
 * reference Plan constructor.  Returns 0 if N is not a power of two. */
int oracle_plan_twiddles(int N, int inverse, float* W_interleaved);

/* Window builder + normaliser (FP64 -> float), fft_cffi.cpp:163-208. */
void oracle_build_window(int kind, int W, float p1, float p2, int norm_policy, float* out);

/* In-place batched transform of X (N x B column-major, interleaved complex),
 * i.e. eigfft::fft_inplace_batched_with_metadata with the context's plan
 * flags.  Returns 1 on success, 0 on a metadata buffer that is too small
 * (the reference throws std::invalid_argument there). */
int oracle_fft_columns(const oracle_cfg* cfg, float* X, size_t B,
                       const oracle_meta_req* reqs, int nreq, int threads);

/* fft_execute_batched (fast path).  Returns frames produced. */
size_t oracle_execute_batched(const oracle_cfg* cfg, const float* pcm, size_t pcm_len,
                              float* out_real, float* out_imag, float* out_mag,
                              int pad_mode, size_t max_frames, int threads);

/* fft_execute_complex_batched (fast path).  Returns frames. */
size_t oracle_execute_complex_batched(const oracle_cfg* cfg, const float* in_real,
                                      const float* in_imag, size_t frames, float* out_pcm,
                                      size_t max_frames, int threads);

/* Frame count rule of fft_execute_batched (fft_cffi.cpp:710-750). */
size_t oracle_frame_count(int N, int window, int hop, int ctx_pad_mode, size_t pcm_len,
                          int pad_mode, size_t max_frames);

#ifdef __cplusplus
}
#endif

#endif
