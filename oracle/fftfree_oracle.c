/*
 * fftfree_oracle.c -- CPU restatement of the fftfree batched STFT/FFT path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): see fftfree_oracle.h.  Every
 * function cites the reference lines it restates.  Arithmetic is float32 in
 * the same operation order as the reference's scalar butterfly path
 * (butterfly_kernel.hpp:91-96, 223-229); built with -ffp-contract=off so the
 * rounding is reproducible.  The reference's own Release build uses
 * -ffast-math -march=native, so it may contract to FMA: results agree to
 * rounding, not bit-for-bit, in the floating-point outputs.  Integer-valued
 * metadata is exact.
 */
#include "fftfree_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float re, im; } cf;

static inline cf cf_mul(cf a, cf b) {
  /* std::complex<float> product as expanded by GCC without NaN recovery. */
  cf r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}
static inline cf cf_add(cf a, cf b) { cf r = {a.re + b.re, a.im + b.im}; return r; }
static inline cf cf_sub(cf a, cf b) { cf r = {a.re - b.re, a.im - b.im}; return r; }
static inline float cf_abs(cf a) { return hypotf(a.re, a.im); }
static inline float cf_norm(cf a) { return a.re * a.re + a.im * a.im; }

static int ilog2_exact(int n) {
  /* Power-of-two check of the Plan constructor (eigen_fft.hpp:2229-2232).
   * The reference loops forever for n == 0; here it is rejected. */
  if (n <= 0) return -1;
  int lg = 0, t = n;
  while ((t & 1) == 0) { ++lg; t >>= 1; }
  return ((1 << lg) == n) ? lg : -1;
}

/* eigen_fft.hpp:2234-2242: tau = sgn * float(2*acos(float(-1))) / float(N),
 * angle = tau * float(k), W[k] = (cosf(angle), sinf(angle)). */
int oracle_plan_twiddles(int N, int inverse, float* W) {
  if (ilog2_exact(N) < 0) return 0;
  const float sgn = inverse ? 1.0f : -1.0f;
  const float two_pi = 2 * acosf(-1.0f);
  const float tau = sgn * two_pi / (float)N;
  for (int k = 0; k < N / 2; ++k) {
    const float ang = tau * (float)k;
    W[2 * k] = cosf(ang);
    W[2 * k + 1] = sinf(ang);
  }
  if (N / 2 == 0) { W[0] = 0.0f; W[1] = 0.0f; }
  return 1;
}

/* fft_cffi.cpp:163-208 (build_window / normalize_window). */
void oracle_build_window(int kind, int W, float p1, float p2, int norm_policy, float* w) {
  (void)p2;
  const double pi = 3.141592653589793238462643383279502884;
  if (W <= 0) return;
  for (int n = 0; n < W; ++n) w[n] = 1.0f;
  switch (kind) {
    case 0: break;
    case 1:
    case 5: /* Kaiser is a Hann placeholder in the reference (fft_cffi.cpp:200-203) */
      for (int n = 0; n < W; ++n) w[n] = (float)(0.5 * (1.0 - cos(2.0 * pi * n / (W - 1))));
      break;
    case 2:
      for (int n = 0; n < W; ++n) w[n] = (float)(0.54 - 0.46 * cos(2.0 * pi * n / (W - 1)));
      break;
    case 3:
      for (int n = 0; n < W; ++n) {
        const double a0 = 0.42, a1 = 0.5, a2 = 0.08;
        w[n] = (float)(a0 - a1 * cos(2.0 * pi * n / (W - 1)) + a2 * cos(4.0 * pi * n / (W - 1)));
      }
      break;
    case 4: {
      const double alpha = (p1 == 0.0f ? 0.5 : p1);
      const int L = (W - 1 > 1) ? W - 1 : 1;
      for (int n = 0; n < W; ++n) {
        const double x = (double)n / (double)L;
        if (x < alpha / 2) w[n] = (float)(0.5 * (1 + cos(pi * (2 * x / alpha - 1))));
        else if (x <= 1 - alpha / 2) w[n] = 1.0f;
        else w[n] = (float)(0.5 * (1 + cos(pi * (2 * x / alpha - 2 / alpha + 1))));
      }
      break;
    }
    default: break;
  }
  if (norm_policy == 1) {
    double s2 = 0.0;
    for (int n = 0; n < W; ++n) s2 += (double)w[n] * (double)w[n];
    s2 = sqrt(s2 > 1e-30 ? s2 : 1e-30);
    if (s2 > 0) for (int n = 0; n < W; ++n) w[n] = (float)(w[n] / s2);
  } else if (norm_policy == 2) {
    double s = 0.0;
    for (int n = 0; n < W; ++n) s += (double)w[n];
    if (fabs(s) > 1e-30) for (int n = 0; n < W; ++n) w[n] = (float)(w[n] / s);
  }
}

static int effective_transform(int t) { return (t >= 0 && t <= 3) ? t : 0; }
static int is_stockham(const oracle_cfg* c) { return c->kernel == 2; }

/* ---------------------------------------------------------------------- */
/* pre/post hooks: eigen_fft.hpp:2484-2596                                 */

static void pre_transform(const oracle_cfg* c, cf* col) {
  const int N = c->N;
  const int mode = effective_transform(c->transform);
  if (mode == 1) {
    for (int i = 0; i < N; ++i) if (col[i].im != 0.0f) col[i].im = 0.0f;
    return;
  }
  if (mode == 2 && c->half_spectrum) {
    if (c->store_polar) {
      for (int k = 0; k <= N / 2; ++k) {
        const float mag = col[k].re, ph = col[k].im;
        col[k].re = mag * cosf(ph);
        col[k].im = mag * sinf(ph);
      }
    }
    col[0].im = 0.0f;
    col[N / 2].im = 0.0f;
    for (int k = 1; k < N / 2; ++k) { col[N - k].re = col[k].re; col[N - k].im = -col[k].im; }
  }
}

static void post_transform(const oracle_cfg* c, cf* col) {
  const int N = c->N;
  const int mode = effective_transform(c->transform);
  const int r2c_half = (mode == 1 && c->half_spectrum);
  if (r2c_half) {
    col[0].im = 0.0f;
    col[N / 2].im = 0.0f;
    for (int k = N / 2 + 1; k < N; ++k) { col[k].re = 0.0f; col[k].im = 0.0f; }
  }
  const int upper = r2c_half ? (N / 2 + 1) : N;
  if (c->store_polar) {
    for (int i = 0; i < upper; ++i) {
      const float mag = cf_abs(col[i]);
      const float ph = atan2f(col[i].im, col[i].re);
      col[i].re = mag; col[i].im = ph;
    }
    return;
  }
  if (c->reduce_magnitude) {
    for (int i = 0; i < upper; ++i) { col[i].re = cf_abs(col[i]); col[i].im = 0.0f; }
    return;
  }
  if (mode == 2) {
    for (int i = 0; i < N; ++i) if (col[i].im != 0.0f) col[i].im = 0.0f;
  }
}

/* ---------------------------------------------------------------------- */
/* metadata lookup                                                         */

typedef struct {
  cf* twiddle; size_t twiddle_n;
  cf* layout; size_t layout_n;
  cf* snap; cf* params; cf* pairs; cf* inv; cf* twmap; cf* omega;
  cf* snap_all; cf* pairs_all; cf* twmap_all;
  int any;
} meta_set;

static int collect_meta(const oracle_cfg* c, size_t B, const oracle_meta_req* reqs, int nreq,
                        meta_set* m) {
  memset(m, 0, sizeof(*m));
  const int N = c->N;
  const int S = ilog2_exact(N);
  const size_t NS = (size_t)N * (size_t)S;
  const int stockham = is_stockham(c);
  int seen[11] = {0};
  for (int i = 0; i < nreq; ++i) {
    const int k = reqs[i].kind;
    cf* buf = (cf*)reqs[i].buf;
    const size_t cnt = reqs[i].count;
    if (k < 0 || k > 10) continue;
    if (k == ORACLE_META_TWIDDLE) {
      /* eigen_fft.hpp:1538-1558: every Twiddle request is validated and the
       * last one is the buffer written (the loop has no break). */
      size_t total = 0;
      for (int s = 0; s < S; ++s) total += (size_t)1 << s;
      if (total > 0 && (!buf || cnt < total)) return 0;
      m->twiddle = buf; m->twiddle_n = total;
      continue;
    }
    if (seen[k]) continue; /* the other writers stop at the first request */
    seen[k] = 1;
    switch (k) {
      case ORACLE_META_LAYOUT_MAP: /* :1604-1619 */
        if (buf && cnt < (size_t)N) return 0;
        m->layout = buf; break;
      case ORACLE_META_STAGE_SNAPSHOT: /* :1637-1649 */
        if (S <= 0) break;
        if (!buf || cnt < NS) return 0;
        m->snap = buf; break;
      case ORACLE_META_STAGE_PARAMS:
        if (S <= 0) break;
        if (!buf || cnt < (size_t)S) return 0;
        m->params = buf; break;
      case ORACLE_META_BUTTERFLY_PAIRS:
        if (S <= 0) break;
        if (!buf || cnt < NS) return 0;
        m->pairs = buf; break;
      case ORACLE_META_STAGE_INVARIANT:
        if (S <= 0) break;
        if (!buf || cnt < (size_t)S) return 0;
        m->inv = buf; break;
      case ORACLE_META_TWIDDLE_INDEX_MAP:
        if (S <= 0) break;
        if (!buf || cnt < NS) return 0;
        m->twmap = buf; break;
      case ORACLE_META_OMEGA: /* :1772-1786; constructed by Cooley-Tukey only */
        if (stockham) break;
        if (buf && cnt < (size_t)N) return 0;
        m->omega = buf;
        break;
      case ORACLE_META_STAGE_SNAPSHOT_ALL:
      case ORACLE_META_BUTTERFLY_PAIRS_ALL:
      case ORACLE_META_TWIDDLE_INDEX_MAP_ALL:
        /* :1809-1888; constructed only by the Cooley-Tukey executor */
        if (stockham || S <= 0 || B == 0) break;
        if (!buf || cnt < NS * B) return 0;
        if (k == ORACLE_META_STAGE_SNAPSHOT_ALL) m->snap_all = buf;
        else if (k == ORACLE_META_BUTTERFLY_PAIRS_ALL) m->pairs_all = buf;
        else m->twmap_all = buf;
        break;
    }
  }
  m->any = (m->twiddle || m->layout || m->snap || m->params || m->pairs || m->inv ||
            m->twmap || m->omega || m->snap_all || m->pairs_all || m->twmap_all);
  return 1;
}

static void record_twiddles(const meta_set* m, int N, int S, const cf* W) {
  /* TwiddleMetadataWriter::record_plan_twiddles (eigen_fft.hpp:1572-1583) */
  if (!m->twiddle) return;
  for (int s = 0; s < S; ++s) {
    const int mm = 1 << s, step = N / (mm << 1);
    for (int j = 0; j < mm; ++j) m->twiddle[(mm - 1) + j] = W[j * step];
  }
}

static void fill_omega(const oracle_cfg* c, cf* omega) {
  /* OmegaMetadataWriter::fill (eigen_fft.hpp:1788-1798) */
  const int N = c->N;
  const int upper = (effective_transform(c->transform) == 1 && c->half_spectrum) ? N / 2 + 1 : N;
  const float two_pi = (float)(2 * acosf(-1.0f));
  for (int k = 0; k < upper; ++k) {
    omega[k].re = two_pi * (float)k / (float)N;
    omega[k].im = 0.0f;
  }
}

/* ---------------------------------------------------------------------- */
/* Cooley-Tukey: eigen_fft.hpp:2655-3100                                   */

static void ct_execute(const oracle_cfg* c, cf* X, size_t B, const meta_set* m, int threads) {
  const int N = c->N;
  const int S = ilog2_exact(N);
  cf* W = (cf*)malloc(sizeof(cf) * (size_t)(N / 2 > 1 ? N / 2 : 1));
  oracle_plan_twiddles(N, c->inverse, (float*)W);
  record_twiddles(m, N, S, W);
  if (m->omega) fill_omega(c, m->omega);

  for (size_t b = 0; b < B; ++b) pre_transform(c, X + b * (size_t)N);
  if (m->layout) for (int p = 0; p < N; ++p) { m->layout[p].re = (float)p; m->layout[p].im = 0.0f; }
  if (m->inv) for (int s = 0; s < S; ++s) { m->inv[s].re = 0.0f; m->inv[s].im = 0.0f; }

  /* bit-reverse swap permutation (:2805-2865) */
  int* bitrev = (int*)malloc(sizeof(int) * (size_t)N);
  for (int i = 0; i < N; ++i) {
    unsigned x = (unsigned)i, r = 0;
    for (int b = 0; b < S; ++b) { r = (r << 1) | (x & 1u); x >>= 1; }
    bitrev[i] = (int)r;
  }
  #pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
  for (long long bb = 0; bb < (long long)B; ++bb) {
    cf* col = X + (size_t)bb * (size_t)N;
    for (int i = 0; i < N; ++i) {
      const int src = bitrev[i];
      if (src <= i) continue;
      cf t = col[i]; col[i] = col[src]; col[src] = t;
    }
  }

  /* stage loop (:2902-3057); each stage is one pass over every column, the
   * reference's per-stage job structure. */
  float* inv_r0 = (float*)calloc((size_t)(S > 0 ? S : 1), sizeof(float));
  float* inv_e = (float*)calloc((size_t)(S > 0 ? S : 1), sizeof(float));
  const int serial = m->any;
  for (int len = 2, s = 0; len <= N; len <<= 1, ++s) {
    const int half = len >> 1, step = N / len, blocks = N / len;
    if (m->params) { m->params[s].re = (float)len; m->params[s].im = (float)step; }
    #pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1 && !serial)
    for (long long bb = 0; bb < (long long)B; ++bb) {
      cf* col = X + (size_t)bb * (size_t)N;
      for (int k = 0; k < half; ++k) {
        const cf w = W[k * step];
        const int tw_index = k * step;
        for (int block = 0; block < blocks; ++block) {
          const int a = block * len + k, b = a + half;
          const cf a_in = col[a], b_in = col[b];
          const cf t = cf_mul(b_in, w);
          const cf y0 = cf_add(a_in, t), y1 = cf_sub(a_in, t);
          col[a] = y0; col[b] = y1;
          if (!serial) continue;
          const size_t bi = (size_t)bb;
          if (m->snap_all) {
            const size_t base = (size_t)s * (size_t)N * B + bi * (size_t)N;
            m->snap_all[base + a] = y0; m->snap_all[base + b] = y1;
          } else if (m->snap && bi == 0) {
            m->snap[(size_t)s * N + a] = y0; m->snap[(size_t)s * N + b] = y1;
          }
          if (m->twmap_all) {
            const size_t base = (size_t)s * (size_t)N * B + bi * (size_t)N;
            cf v = {(float)tw_index, 0.0f};
            m->twmap_all[base + a] = v; m->twmap_all[base + b] = v;
          } else if (m->twmap && bi == 0) {
            cf v = {(float)tw_index, 0.0f};
            m->twmap[(size_t)s * N + a] = v; m->twmap[(size_t)s * N + b] = v;
          }
          if (m->inv) {
            const cf sum = cf_add(y0, y1);
            cf two_a = {2.0f * a_in.re, 2.0f * a_in.im};
            const float r0 = cf_abs(cf_sub(sum, two_a));
            const float e = (cf_norm(y0) + cf_norm(y1)) - 2.0f * (cf_norm(a_in) + cf_norm(b_in));
            const float ae = fabsf(e);
            if (r0 > inv_r0[s]) inv_r0[s] = r0;
            if (ae > inv_e[s]) inv_e[s] = ae;
          }
          if (m->pairs_all) {
            const size_t base = (size_t)s * (size_t)N * B + bi * (size_t)N;
            cf v = {(float)a, (float)b};
            m->pairs_all[base + a] = v; m->pairs_all[base + b] = v;
          } else if (m->pairs && bi == 0) {
            cf v = {(float)a, (float)b};
            m->pairs[(size_t)s * N + a] = v; m->pairs[(size_t)s * N + b] = v;
          }
        }
      }
    }
  }
  if (m->inv) for (int s = 0; s < S; ++s) { m->inv[s].re = inv_r0[s]; m->inv[s].im = inv_e[s]; }

  if (c->inverse) { /* :3076-3085 */
    const float scale = 1.0f / (float)N;
    for (size_t i = 0; i < (size_t)N * B; ++i) { X[i].re *= scale; X[i].im *= scale; }
  }
  for (size_t b = 0; b < B; ++b) post_transform(c, X + b * (size_t)N);
  free(inv_r0); free(inv_e); free(bitrev); free(W);
}

/* ---------------------------------------------------------------------- */
/* Stockham: eigen_fft.hpp:3227-3623 (one column per chunk)                */

static void stockham_execute(const oracle_cfg* c, cf* X, size_t B, const meta_set* m, int threads) {
  const int N = c->N;
  const int S = ilog2_exact(N);
  if (m->layout) for (int p = 0; p < N; ++p) { m->layout[p].re = (float)p; m->layout[p].im = 0.0f; }
  if (m->inv) for (int s = 0; s < S; ++s) { m->inv[s].re = 0.0f; m->inv[s].im = 0.0f; }
  if (B == 0) return;
  cf* W = (cf*)malloc(sizeof(cf) * (size_t)(N / 2 > 1 ? N / 2 : 1));
  oracle_plan_twiddles(N, c->inverse, (float*)W);
  record_twiddles(m, N, S, W);

  float* inv_r0 = (float*)calloc((size_t)(S > 0 ? S : 1), sizeof(float));
  float* inv_e = (float*)calloc((size_t)(S > 0 ? S : 1), sizeof(float));
  const int serial = m->any;
  #pragma omp parallel num_threads(threads) if (threads > 1 && !serial)
  {
    cf* ping = (cf*)malloc(sizeof(cf) * (size_t)N);
    cf* pong = (cf*)malloc(sizeof(cf) * (size_t)N);
    #pragma omp for schedule(static)
    for (long long bb = 0; bb < (long long)B; ++bb) {
      cf* col = X + (size_t)bb * (size_t)N;
      const int capture = (bb == 0) && serial;
      memcpy(ping, col, sizeof(cf) * (size_t)N);
      cf* in = ping; cf* out = pong;
      for (int s = 0; s < S; ++s) {
        const int mm = 1 << s, distance = mm << 1, seg = N >> (s + 1), halfN = N >> 1;
        if (capture && m->params) { m->params[s].re = (float)distance; m->params[s].im = (float)seg; }
        for (int j = 0; j < mm; ++j) {
          const int tw_index = j * seg;
          const cf w = W[tw_index];
          for (int g = 0; g < seg; ++g) {
            const int i0 = 2 * j * seg + g, i1 = i0 + seg;
            const int o0 = j * seg + g, o1 = o0 + halfN;
            const cf a_in = in[i0], b_in = in[i1];
            const cf t = cf_mul(b_in, w);
            const cf y0 = cf_add(a_in, t), y1 = cf_sub(a_in, t);
            out[o0] = y0; out[o1] = y1;
            if (!serial) continue;
            if (capture && m->pairs) {
              cf v = {(float)i0, (float)i1};
              m->pairs[(size_t)s * N + o0] = v; m->pairs[(size_t)s * N + o1] = v;
            }
            if (capture && m->twmap) {
              cf v = {(float)tw_index, 0.0f};
              m->twmap[(size_t)s * N + o0] = v; m->twmap[(size_t)s * N + o1] = v;
            }
            if (m->inv) {
              const cf sum = cf_add(y0, y1);
              cf two_a = {2.0f * a_in.re, 2.0f * a_in.im};
              const float r0 = cf_abs(cf_sub(sum, two_a));
              const float e = (cf_norm(y0) + cf_norm(y1)) - 2.0f * (cf_norm(a_in) + cf_norm(b_in));
              const float ae = fabsf(e);
              if (r0 > inv_r0[s]) inv_r0[s] = r0;
              if (ae > inv_e[s]) inv_e[s] = ae;
            }
          }
        }
        if (capture && m->snap) for (int i = 0; i < N; ++i) m->snap[(size_t)s * N + i] = out[i];
        cf* t = in; in = out; out = t;
      }
      /* final buffer: stages even -> ping, odd -> pong (== `in` here) */
      if (c->inverse) {
        const float scale = 1.0f / (float)N;
        for (int i = 0; i < N; ++i) { col[i].re = in[i].re * scale; col[i].im = in[i].im * scale; }
      } else {
        memcpy(col, in, sizeof(cf) * (size_t)N);
      }
    }
    free(ping); free(pong);
  }
  if (m->inv) for (int s = 0; s < S; ++s) { m->inv[s].re = inv_r0[s]; m->inv[s].im = inv_e[s]; }
  for (size_t b = 0; b < B; ++b) post_transform(c, X + b * (size_t)N);
  free(inv_r0); free(inv_e); free(W);
}

int oracle_fft_columns(const oracle_cfg* c, float* X, size_t B,
                       const oracle_meta_req* reqs, int nreq, int threads) {
  if (ilog2_exact(c->N) < 0) return 0;
  meta_set m;
  if (!collect_meta(c, B, reqs, nreq, &m)) return 0;
  if (threads < 1) threads = 1;
  if (is_stockham(c)) stockham_execute(c, (cf*)X, B, &m, threads);
  else ct_execute(c, (cf*)X, B, &m, threads);
  return 1;
}

/* ---------------------------------------------------------------------- */
/* fft_execute_batched: fft_cffi.cpp:701-1034 (fast path)                  */

size_t oracle_frame_count(int N, int window, int hop, int ctx_pad_mode, size_t pcm_len,
                          int pad_mode, size_t max_frames) {
  if (N <= 0 || pcm_len == 0) return 0;
  const int W = window ? window : N;
  const int H = hop ? hop : W;
  if (W <= 0 || H <= 0) return 0;
  if (W > N) return 0;
  const int eff = (pad_mode == 0) ? ctx_pad_mode : pad_mode;
  size_t frames = 0;
  if (pcm_len < (size_t)W) {
    if (eff == 1) frames = 1; else return 0;
  } else {
    frames = 1 + (pcm_len - (size_t)W) / (size_t)H;
    const size_t last = (frames - 1) * (size_t)H;
    const size_t remaining = (pcm_len > last) ? pcm_len - last : 0;
    if (remaining < (size_t)W) {
      if (eff == 1) { }
      else if (eff == 2) { if (frames > 0) frames -= 1; }
      else return 0;
    }
  }
  if (frames == 0) return 0;
  if (max_frames != 0 && frames > max_frames) frames = max_frames;
  return frames;
}

size_t oracle_execute_batched(const oracle_cfg* c, const float* pcm, size_t pcm_len,
                              float* out_real, float* out_imag, float* out_mag,
                              int pad_mode, size_t max_frames, int threads) {
  if (!pcm || pcm_len == 0 || !out_real || !out_imag || !out_mag) return 0;
  const int N = c->N;
  if (N <= 0) return 0;
  const int W = c->window ? c->window : N;
  const int H = c->hop ? c->hop : W;
  const size_t frames = oracle_frame_count(N, c->window, c->hop, c->pad_mode, pcm_len, pad_mode, max_frames);
  if (frames == 0) return 0;
  const size_t plan_n = (size_t)N;
  /* 64 MiB column batches (:754-758) */
  const size_t max_bytes = 64ull * 1024ull * 1024ull;
  size_t batch = max_bytes / (plan_n * sizeof(cf) + 1);
  if (batch < 1) batch = 1;
  if (batch > frames) batch = frames;
  cf* buf = (cf*)malloc(sizeof(cf) * plan_n * batch);
  const size_t bins = c->half_spectrum ? plan_n / 2 + 1 : plan_n;
  if (threads < 1) threads = 1;
  for (size_t b0 = 0; b0 < frames; b0 += batch) {
    const size_t cnt = (frames - b0 < batch) ? frames - b0 : batch;
    /* framing (:765-791) */
    #pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
    for (long long ff = 0; ff < (long long)cnt; ++ff) {
      const size_t f = (size_t)ff;
      const size_t start = (b0 + f) * (size_t)H;
      size_t copy = 0;
      if (start < pcm_len) copy = ((size_t)W < pcm_len - start) ? (size_t)W : pcm_len - start;
      cf* col = buf + f * plan_n;
      const int win = c->windows_enabled && c->analysis_win;
      for (size_t i = 0; i < copy; ++i) {
        col[i].re = win ? pcm[start + i] * c->analysis_win[i] : pcm[start + i];
        col[i].im = 0.0f;
      }
      for (size_t i = copy; i < plan_n; ++i) { col[i].re = 0.0f; col[i].im = 0.0f; }
    }
    oracle_fft_columns(c, (float*)buf, cnt, NULL, 0, threads);
    /* output copy (:813-824) */
    #pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
    for (long long ff = 0; ff < (long long)cnt; ++ff) {
      const size_t f = (size_t)ff;
      const size_t ob = (b0 + f) * bins;
      const cf* col = buf + f * plan_n;
      for (size_t i = 0; i < bins; ++i) {
        out_real[ob + i] = col[i].re;
        out_imag[ob + i] = col[i].im;
        out_mag[ob + i] = c->store_polar ? col[i].re : cf_abs(col[i]);
      }
    }
  }
  free(buf);
  return frames;
}

/* ---------------------------------------------------------------------- */
/* fft_execute_complex_batched: fft_cffi.cpp:1042-1340 (fast path)         */

static float cola_weight(const oracle_cfg* c, int i) {
  /* fft_cffi.cpp:210-226 */
  if (!c->windows_enabled) return 1.0f;
  const float a = c->analysis_win ? c->analysis_win[i] : 1.0f;
  const float s = c->synthesis_win ? c->synthesis_win[i] : 1.0f;
  return a * s;
}

size_t oracle_execute_complex_batched(const oracle_cfg* c, const float* in_real,
                                      const float* in_imag, size_t frames, float* out_pcm,
                                      size_t max_frames, int threads) {
  if (!in_real || !in_imag || !out_pcm || frames == 0) return 0;
  const int N = c->N;
  if (N <= 0) return 0;
  const size_t plan_n = (size_t)N;
  const size_t bins = c->half_spectrum ? plan_n / 2 + 1 : plan_n;
  if (max_frames != 0 && frames > max_frames) frames = max_frames;
  if (threads < 1) threads = 1;
  cf* buf = (cf*)malloc(sizeof(cf) * plan_n * frames);
  const int c2r_half = c->half_spectrum && effective_transform(c->transform) == 2;
  #pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
  for (long long ff = 0; ff < (long long)frames; ++ff) {
    const size_t f = (size_t)ff;
    cf* col = buf + f * plan_n;
    for (size_t i = 0; i < bins; ++i) { col[i].re = in_real[f * bins + i]; col[i].im = in_imag[f * bins + i]; }
    if (c2r_half) {
      col[0].im = 0.0f;
      const size_t ny = plan_n / 2;
      if (ny < bins) col[ny].im = 0.0f;
      const size_t maxk = (bins > ny + 1) ? ny : bins - 1;
      for (size_t k = 1; k < maxk; ++k) { col[plan_n - k].re = col[k].re; col[plan_n - k].im = -col[k].im; }
    } else {
      for (size_t i = bins; i < plan_n; ++i) { col[i].re = 0.0f; col[i].im = 0.0f; }
    }
  }
  oracle_fft_columns(c, (float*)buf, frames, NULL, 0, threads);
  const int win = c->windows_enabled && c->synthesis_win;
  if (c->apply_ola) {
    const int H = (c->hop > 0) ? c->hop : ((c->window > 0) ? c->window : N);
    const size_t total = frames * plan_n;
    for (size_t t = 0; t < total; ++t) out_pcm[t] = 0.0f;
    float* norm = (c->cola_mode == 1) ? (float*)calloc(total, sizeof(float)) : NULL;
    for (size_t f = 0; f < frames; ++f) {
      const cf* col = buf + f * plan_n;
      const size_t start = f * (size_t)H;
      for (size_t i = 0; i < plan_n; ++i) {
        float s = col[i].re;
        if (win) s *= c->synthesis_win[i];
        const size_t t = start + i;
        if (t < total) {
          out_pcm[t] += s;
          if (norm) norm[t] += cola_weight(c, (int)i);
        }
      }
    }
    if (norm) {
      for (size_t t = 0; t < total; ++t) if (norm[t] > 1e-12f) out_pcm[t] /= norm[t];
      free(norm);
    }
  } else {
    #pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
    for (long long ff = 0; ff < (long long)frames; ++ff) {
      const size_t f = (size_t)ff;
      const cf* col = buf + f * plan_n;
      for (size_t i = 0; i < plan_n; ++i) {
        float s = col[i].re;
        if (win) s *= c->synthesis_win[i];
        out_pcm[f * plan_n + i] = s;
      }
    }
  }
  free(buf);
  return frames;
}
