// io.cuh -- per-path load/store policies of the FFT kernels (device code):
// STFT framing + real-input untangle epilogue, complex C2C with the plan's
// hooks, complex/inverse batch, Hermitian C2R half-size path.  Each policy
// also provides elem4/emit4 (one input element / one output bin by index)
// for the multi-pass kernels.
#pragma once

#include <stdint.h>

#include <type_traits>

#include "fft_engine.cuh"
#include "kernels.h"

namespace ffb {
// ------------------------------------------------------------------ hooks
// |z| as sqrt(x^2 + y^2): the squares summed with one rounding (fma), then
// s * rsqrt(s) (the hardware reciprocal square root and one multiply, a few
// ulp) while s is a normal float away from overflow; zero, tiny and huge
// magnitudes through hypotf.
__device__ __forceinline__ float cabs_fast(float x, float y) {
  const float s = __fmaf_rn(x, x, __fmul_rn(y, y));
  if (s > 1e-36f && s < 1e36f) return __fmul_rn(s, rsqrtf(s));
  return hypotf(x, y);
}

__device__ __forceinline__ bool any_post(const PostFlags& pf) {
  return (pf.r2c_half | pf.polar | pf.reduce | pf.clear_imag) != 0;
}

// Phase and polar conversions of the hooks, written for throughput: the
// polar epilogues spend most of their instructions here.
//
// atan2: octant reduction to a = min(|x|,|y|) / max(|x|,|y|) in [0, 1],
// atan(a) = a P(a^2) with P of degree 7 fitted to atan on [0, 1] (weighted
// least squares on Chebyshev nodes, coefficients rounded to float: 9.2e-8
// rad), then pi/2 - r, pi - r and the sign of y as the octant says; C's
// atan2 results for zero arguments.  Max error against FP64: 3.6e-7 rad.
__device__ __forceinline__ float atan2_fast(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  if (mx > 1e30f || mx < 1e-30f) {  // keep the fast division in its range
    const float sc = (mx > 1e30f) ? 0x1p-64f : 0x1p64f;
    mx *= sc;
    mn *= sc;
  }
  // both zero: a = 0, which the octant steps below turn into C's atan2 of
  // signed zeros (0, or pi for x = -0, with the sign of y)
  const float a = (mx > 0.f) ? __fdividef(mn, mx) : 0.f;
  const float t = a * a;
  float p = -0.004780322778970003f;
  p = fmaf(p, t, 0.024556664749979973f);
  p = fmaf(p, t, -0.05990409106016159f);
  p = fmaf(p, t, 0.09942717105150223f);
  p = fmaf(p, t, -0.14029406011104584f);
  p = fmaf(p, t, 0.19971372187137604f);
  p = fmaf(p, t, -0.3333209455013275f);
  p = fmaf(p, t, 0.9999999403953552f);
  float r = a * p;
  if (ay > ax) r = 1.5707963705062866f - r;
  if (signbit(x)) r = 3.1415927410125732f - r;
  return copysignf(r, y);
}

// sin and cos: Cody-Waite reduction by pi/2 split into three floats (with
// FMA, exact to the float rounding of r for |x| <= 8192) to |r| <= pi/4,
// sin(r) = r Q(r^2) and cos(r) = P(r^2) with Q of degree 3 and P of degree 4
// fitted to sin(r)/r and cos(r) on [0, pi/4] (max 4e-9), the quadrant
// swapping and negating them; larger |x| (and NaN) through sincosf.  Max
// error against FP64: 8.7e-8.
__device__ __forceinline__ void sincos_fast(float x, float* sn, float* cs) {
  if (!(fabsf(x) <= 8192.f)) {
    sincosf(x, sn, cs);
    return;
  }
  const float k = rintf(x * 0.6366197466850281f);
  float r = fmaf(-k, 1.5707963705062866f, x);
  r = fmaf(-k, -4.371138828673793e-08f, r);
  r = fmaf(-k, -1.7151245100058819e-15f, r);
  const float t = r * r;
  float q = -0.00019504022202454507f;
  q = fmaf(q, t, 0.008332036435604095f);
  q = fmaf(q, t, -0.16666650772094727f);
  q = fmaf(q, t, 1.0f);
  const float s0 = r * q;
  float c = 2.4379929527640343e-05f;
  c = fmaf(c, t, -0.0013886619126424193f);
  c = fmaf(c, t, 0.04166661575436592f);
  c = fmaf(c, t, -0.5f);
  const float c0 = fmaf(c, t, 1.0f);
  const int quad = (int)k & 3;
  const float ss = (quad & 1) ? c0 : s0;
  const float cc = (quad & 1) ? s0 : c0;
  *sn = (quad & 2) ? -ss : ss;
  *cs = ((quad + 1) & 2) ? -cc : cc;
}

__device__ __forceinline__ float2 post_hook(float2 X, int k, int N, const PostFlags& pf) {
  // eigen_fft.hpp:2544-2595.  Polar/reduce apply below `upper`; above it the
  // R2C half branch has already zeroed the value, and (0,0) is a fixed point
  // of both, so applying them everywhere is equivalent.
  if (pf.r2c_half) {
    if (k > (N >> 1)) X = make_float2(0.f, 0.f);
    else if (k == 0 || k == (N >> 1)) X.y = 0.f;
  }
  if (pf.polar) {
    const float m = cabs_fast(X.x, X.y);
    const float ph = atan2_fast(X.y, X.x);
    X = make_float2(m, ph);
  } else if (pf.reduce) {
    X = make_float2(cabs_fast(X.x, X.y), 0.f);
  } else if (pf.clear_imag) {
    X.y = 0.f;
  }
  return X;
}

// (m, phi) -> m e^{i phi}.  Phases in [-pi, pi] (those atan2 produces) use
// the hardware sine / cosine (absolute error below 2^-21 there); others go
// through sincos_fast.
__device__ __forceinline__ float2 polar_to_complex(float2 u) {
  float s, c;
  if (fabsf(u.y) <= 3.14159274f) {
    __sincosf(u.y, &s, &c);
  } else {
    sincos_fast(u.y, &s, &c);
  }
  return make_float2(u.x * c, u.x * s);
}

__device__ __forceinline__ bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7) == 0; }

// Post-hook with the polar / magnitude choice fixed at compile time
// (MODE 0: none or imag clear, 1: reduce_magnitude, 2: store_polar), so an
// unrolled epilogue carries only the arithmetic it needs.
template <int MODE>
__device__ __forceinline__ float2 post_hook_m(float2 X, int k, int N, const PostFlags& pf) {
  if (pf.r2c_half) {
    if (k > (N >> 1)) X = make_float2(0.f, 0.f);
    else if (k == 0 || k == (N >> 1)) X.y = 0.f;
  }
  if constexpr (MODE == 2) return make_float2(cabs_fast(X.x, X.y), atan2_fast(X.y, X.x));
  if constexpr (MODE == 1) return make_float2(cabs_fast(X.x, X.y), 0.f);
  if (pf.clear_imag) X.y = 0.f;
  return X;
}

__host__ __device__ inline int post_mode(const PostFlags& pf) { return pf.polar ? 2 : (pf.reduce ? 1 : 0); }

// X / |X| for the magnitude gradient's saved phasor; 0 where |X| = 0, where
// the gradient of |X| is taken as 0.  X * rsqrt(|X|^2) (a few ulp, far inside
// the gradient's tolerance) in the range where |X|^2 is a normal float.
__device__ __forceinline__ float2 unit_phasor(float2 X, float mag) {
  if (!(mag > 0.f)) return make_float2(0.f, 0.f);
  const float s = fmaf(X.x, X.x, X.y * X.y);
  const float r = (s > 1e-36f && s < 1e36f) ? rsqrtf(s) : 1.0f / mag;
  return make_float2(X.x * r, X.y * r);
}

// |X| and X / |X| from one reciprocal square root (cabs_fast's magnitude,
// unit_phasor's phasor, bit for bit).
__device__ __forceinline__ float2 mag_phasor(float2 X, float* mag) {
  const float s = __fmaf_rn(X.x, X.x, __fmul_rn(X.y, X.y));
  if (s > 1e-36f && s < 1e36f) {
    const float r = rsqrtf(s);
    *mag = __fmul_rn(s, r);
    return make_float2(X.x * r, X.y * r);
  }
  const float m = hypotf(X.x, X.y);
  *mag = m;
  return unit_phasor(X, m);
}

// Griffin-Lim projection (phase_infer.hpp:190-196): the magnitude m with the
// phase of X, m e^{i atan2(X.y, X.x)}, formed as m X / |X|.  X = 0 takes
// atan2's phase of signed zeros: 0, or pi where X.x is -0 (cos = -1; the
// sine's 8.7e-8 is left out).
__device__ __forceinline__ float2 gl_project(float2 X, float m) {
  const float s = __fmaf_rn(X.x, X.x, __fmul_rn(X.y, X.y));
  float r;
  if (s > 1e-36f && s < 1e36f) {
    r = m * rsqrtf(s);
  } else {
    const float h = hypotf(X.x, X.y);
    if (h == 0.f) return make_float2(signbit(X.x) ? -m : m, 0.f);
    r = m / h;
  }
  return make_float2(X.x * r, X.y * r);
}

// Frame f of a (possibly multi-signal) STFT: its first sample and how many
// samples it takes from the signal (fft_cffi.cpp:765-791: frame f covers
// pcm[f*H .. f*H + W), zero beyond the signal end and from W up to N).
__device__ __forceinline__ const float* stft_frame(const float* pcm, long long pcm_len, long long sig_frames,
                                                   long long sig_stride, int W, int H, long long f,
                                                   long long* cnt) {
  if (sig_frames > 0) {
    const long long s = f / sig_frames;
    pcm += s * sig_stride;
    f -= s * sig_frames;
  }
  const long long start = f * (long long)H;
  long long c = pcm_len - start;
  if (c > W) c = W;
  *cnt = c;
  return pcm + start;
}

// Slots of squared-residual partial sums per frame of an L2-loss STFT of
// M = N/2 complex points: one per warp of the widest transform group
// (T = M / 4 threads), at least one.
__host__ __device__ constexpr int loss_slots(int M) { return M / 128 > 1 ? M / 128 : 1; }

// Sum of v over the T threads of one transform group, into slots
// part[0 .. loss_slots(M)) of its frame: one sum per warp (or per group when
// T < 32), in a fixed order; unused slots are zeroed.  Every thread of the
// group calls it.
template <class S>
__device__ __forceinline__ void group_loss_partial(float v, int t, float* part) {
  constexpr int T = S::T;
  constexpr int W = T < 32 ? T : 32;
  constexpr int P = T / 32 > 1 ? T / 32 : 1;
  constexpr int SLOTS = loss_slots(S::M);
  const unsigned lane = threadIdx.x & 31u;
  const unsigned mask = (W == 32) ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(unsigned)(W - 1)));
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, W);
  if ((t & (W - 1)) == 0) part[t / W] = v;
  if (t == 0) {
#pragma unroll
    for (int p = P; p < SLOTS; ++p) part[p] = 0.f;
  }
}

// ------------------------------------------------------------------ STFT IO
// MODE: 0 plain / imag clear, 1 reduce_magnitude, 2 store_polar, 3 |X| only
// (forward half spectrum, magnitude array alone), 4 |X| into the magnitude
// array and the unit phasor X / |X| into out_phasor (0 where |X| = 0), 5 the
// residual |X| - target into the magnitude array, the unit phasor, and the
// frame's sum of squared residuals (loss_part, loss_slots per frame), 6 the
// Griffin-Lim projection: mode 0's (re, im) replaced by target e^{i arg}
// (target: the magnitudes, same layout as out_re; no magnitude array).
template <int MODE>
struct StftIO {
  StftArgs a;
  int logN;
  // modes that write the magnitude array alone or with a phasor row
  static constexpr bool kMagOnly = MODE >= 3 && MODE <= 5;
  static constexpr bool kPhasor = MODE == 4 || MODE == 5;
  // modes that read the target row (through the `mg` row pointer in mode 6)
  static constexpr bool kTarget = MODE == 5 || MODE == 6;

  // Row of the magnitude array at offset ob; in mode 6, the target's row
  // (read, never written).
  __device__ __forceinline__ float* mag_row(long long ob) const {
    if constexpr (MODE == 6) return const_cast<float*>(a.target) + ob;
    return a.out_mag + ob;
  }

  template <class S>
  __device__ __forceinline__ void load(long long f, int t, float2 (&v)[S::R], float2*, const Twiddles&) const {
    if (f >= a.frames) {
#pragma unroll
      for (int i = 0; i < S::R; ++i) v[i] = make_float2(0.f, 0.f);
      return;
    }
    // Cooley-Tukey C2R half adds the pre-hook's mirror (eigen_fft.hpp:2523-2528),
    // x[N-n] = x[n] on real frames.
    long long cnt;
    const float* src = stft_frame(a.pcm, a.pcm_len, a.sig_frames, a.sig_stride, a.W, a.H, f, &cnt);
    if (a.N == 1) {
      const float s = (cnt > 0) ? __ldg(src) : 0.f;
#pragma unroll
      for (int i = 0; i < S::R; ++i) v[i] = make_float2(a.win && cnt > 0 ? s * __ldg(a.win) : s, 0.f);
      return;
    }
    if (!a.mirror && cnt == a.N && aligned8(src) && (!a.win || aligned8(a.win))) {
      // whole frame present: z[m] = (x[2m], x[2m+1]) as one 8-byte load
      const float2* s2 = reinterpret_cast<const float2*>(src);
      const float2* w2 = reinterpret_cast<const float2*>(a.win);
#pragma unroll
      for (int i = 0; i < S::R; ++i) {
        const int m = t + i * S::T;
        float2 z = __ldg(s2 + m);
        if (w2) z = __fmul2_rn(z, __ldg(w2 + m));
        v[i] = z;
      }
      return;
    }
    const int half = a.N >> 1;
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int m = t + i * S::T;
      float x[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        int n = 2 * m + j;
        if (a.mirror && n > half) n = a.N - n;
        float s = 0.f;
        if ((long long)n < cnt) {
          s = __ldg(src + n);
          if (a.win) s *= __ldg(a.win + n);
        }
        x[j] = s;
      }
      v[i] = make_float2(x[0], x[1]);
    }
  }

  // Multi-pass access: input element n of frame f as a complex value (the
  // frame is real), and output bin k of the N-point transform.
  __device__ __forceinline__ float2 elem4(long long f, long long n) const {
    if (f >= a.frames) return make_float2(0.f, 0.f);
    int nn = (int)n;
    if (a.mirror && nn > (a.N >> 1)) nn = a.N - nn;
    long long cnt;
    const float* src = stft_frame(a.pcm, a.pcm_len, a.sig_frames, a.sig_stride, a.W, a.H, f, &cnt);
    if ((long long)nn >= cnt) return make_float2(0.f, 0.f);
    float s = __ldg(src + nn);
    if (a.win) s *= __ldg(a.win + nn);
    return make_float2(s, 0.f);
  }
  __device__ __forceinline__ void emit4(long long f, long long k, float2 X) const {
    if (f >= a.frames || k >= a.out_bins) return;
    const long long ob = f * a.out_stride;
    const bool mag_is_re = (MODE == 1) || (MODE == 2 && a.mag_from_real);
    emit(MODE == 4 ? reinterpret_cast<float*>(a.out_phasor + ob) : a.out_re + (MODE == 3 ? 0 : ob),
         a.out_im + (kMagOnly ? 0 : ob), mag_row(ob), (int)k, X, k == 0 || 2 * k == a.N,
         1.0f / (float)a.N, mag_is_re);
  }

  // Bin k of the output: inverse scaling, exact-real DC / Nyquist, post
  // hook, and the three planar stores (fft_cffi.cpp:813-824).
  __device__ __forceinline__ void emit(float* re, float* im, float* mg, int k, float2 X, bool dc_or_nyq,
                                       float inv_n, bool mag_is_re) const {
    if (a.inverse) X = make_float2(X.x * inv_n, -X.y * inv_n);
    // Real input: DC and Nyquist are exactly real (imag +0), as in the
    // reference's radix-2 executors.
    if (dc_or_nyq) X.y = 0.f;
    if constexpr (MODE == 6) {
      X = post_hook_m<0>(X, k, a.N, a.pf);
      const float2 P = gl_project(X, mg[k]);  // mg: the target row
      re[k] = P.x;
      im[k] = P.y;
      return;
    }
    if constexpr (kMagOnly) {
      const float m = cabs_fast(X.x, X.y);
      mg[k] = m;
      if constexpr (MODE == 4) reinterpret_cast<float2*>(re)[k] = unit_phasor(X, m);  // re: phasor row
      return;
    }
    X = post_hook_m<MODE>(X, k, a.N, a.pf);
    re[k] = X.x;
    im[k] = X.y;
    mg[k] = mag_is_re ? X.x : cabs_fast(X.x, X.y);
  }

  template <class S>
  __device__ __forceinline__ void store(long long f, int t, float2 (&v)[S::R], float2* sm,
                                        const Twiddles& tw) const {
    constexpr int M = S::M, T = S::T, R = S::R;
    // L2 loss and projection: the frame's target row (bins 0..M) is fetched
    // first, so that its loads are in flight across the tile exchange
    float tgv[kTarget ? R : 1];
    float tg_nyq = 0.f;
    if constexpr (kTarget) {
      const bool okf = f < a.frames && a.out_bins == M + 1 && !a.inverse;
      const float* tg = a.target + (okf ? f : 0) * a.out_stride + t;
#pragma unroll
      for (int i = 0; i < R; ++i) tgv[i] = okf ? __ldg(tg + i * T) : 0.f;
      if (t == 0 && okf) tg_nyq = __ldg(a.target + f * a.out_stride + M);
    }
    tile_write_natural<S>(v, t, sm);
    GroupSync::sync<S>();
    if (f >= a.frames) return;
    const long long ob = f * a.out_stride;
    float* re = kPhasor ? reinterpret_cast<float*>(a.out_phasor + ob) : a.out_re + (MODE == 3 ? 0 : ob);
    float* im = a.out_im + (kMagOnly ? 0 : ob);
    float* mg = mag_row(ob);
    const bool mag_is_re = (MODE == 1) || (MODE == 2 && a.mag_from_real);
    if (a.N == 1) {
      if (t == 0) emit(re, im, mg, 0, make_float2(v[0].x, 0.f), true, 1.0f, mag_is_re);
      return;
    }
    constexpr int LN = S::LOGM + 1;  // N = 2M
    const float inv_n = 1.0f / (float)(2 * M);
    const int bins = a.out_bins;
    if (bins == M + 1 && !a.inverse) {
      // Common STFT case (half spectrum, forward): bins 0..M, each written
      // once, no bounds or mirror logic.
      const UntangleTw<S> w(tw, t);
      float* pr = re + t;
      float* pi = im + t;
      float* pm = mg + t;
      if constexpr (MODE == 5) {
        float2* ph = reinterpret_cast<float2*>(re) + t;
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const float2 zm = sm[pidx((M - t - i * T) & (M - 1))];
          float2 X = untangle_bin(v[i], zm, w.half(i));
          if (i == 0 && t == 0) X.y = 0.f;  // DC
          float m;
          ph[i * T] = mag_phasor(X, &m);
          const float r = m - tgv[i];
          pm[i * T] = r;
          acc = __fmaf_rn(r, r, acc);
        }
        if (t == 0) {  // Nyquist X[M] = Re Z[0] - Im Z[0]
          float m;
          reinterpret_cast<float2*>(re)[M] = mag_phasor(make_float2(v[0].x - v[0].y, 0.f), &m);
          const float r = m - tg_nyq;
          mg[M] = r;
          acc = __fmaf_rn(r, r, acc);
        }
        group_loss_partial<S>(acc, t, a.loss_part + f * loss_slots(M));
        return;
      }
      if constexpr (MODE == 6) {
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const float2 zm = sm[pidx((M - t - i * T) & (M - 1))];
          float2 X = untangle_bin(v[i], zm, w.half(i));
          if ((i == 0 && t == 0) || a.pf.clear_imag) X.y = 0.f;  // DC is real
          const float2 P = gl_project(X, tgv[i]);
          pr[i * T] = P.x;
          pi[i * T] = P.y;
        }
        if (t == 0) {  // Nyquist X[M] = Re Z[0] - Im Z[0]
          const float2 P = gl_project(make_float2(v[0].x - v[0].y, 0.f), tg_nyq);
          re[M] = P.x;
          im[M] = P.y;
        }
        return;
      }
      // store_polar's magnitude array: |X| itself when it mirrors the real
      // output (fft_execute_batched), else |(|X|, arg X)| -- a uniform
      // choice, taken once outside the unrolled loop
      const auto bins_loop = [&](auto mag_re) {
#pragma unroll
        for (int i = 0; i < R; ++i) {
          const float2 zm = sm[pidx((M - t - i * T) & (M - 1))];
          float2 X = untangle_bin(v[i], zm, w.half(i));
          if (i == 0 && t == 0) X.y = 0.f;  // DC
          if constexpr (MODE == 4) {
            float m;
            reinterpret_cast<float2*>(re)[t + i * T] = mag_phasor(X, &m);
            pm[i * T] = m;
            continue;
          }
          if constexpr (MODE == 3) {
            pm[i * T] = cabs_fast(X.x, X.y);
            continue;
          }
          float mag;
          if constexpr (MODE == 2) {
            mag = cabs_fast(X.x, X.y);
            X = make_float2(mag, atan2_fast(X.y, X.x));
            if constexpr (!decltype(mag_re)::value) mag = cabs_fast(X.x, X.y);
          } else if constexpr (MODE == 1) {
            mag = cabs_fast(X.x, X.y);
            X = make_float2(mag, 0.f);
          } else {
            if (a.pf.clear_imag) X.y = 0.f;
            mag = cabs_fast(X.x, X.y);
          }
          pr[i * T] = X.x;
          pi[i * T] = X.y;
          pm[i * T] = mag;
        }
      };
      if constexpr (MODE == 2) {
        if (a.mag_from_real) bins_loop(std::true_type{});
        else bins_loop(std::false_type{});
      } else {
        bins_loop(std::true_type{});
      }
      if (t == 0) emit(re, im, mg, M, make_float2(v[0].x - v[0].y, 0.f), true, inv_n, mag_is_re);
      return;
    }
    // Real-input untangle of the M-point transform Z of z[m] = x[2m] + i x[2m+1]:
    // X[k] = E + w^k O,  E = (Z[k] + conj Z[M-k]) / 2,  O = -i (Z[k] - conj Z[M-k]) / 2.
    // This thread holds Z[k] for k = t + i*T in v[i]; X[N-k] = conj X[k].
    const float2* w = tw.pyr + ((1 << LN) - 1) + t;
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int k = t + i * T;
      const float2 zk = v[i];
      const float2 zm = sm[pidx((M - k) & (M - 1))];
      const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      const float2 D = make_float2(zk.x - zm.x, zk.y + zm.y);
      const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
      const float2 X = cadd(E, cmul(__ldg(w + i * T), O));
      if (k < bins) emit(re, im, mg, k, X, k == 0, inv_n, mag_is_re);
      if (k > 0 && 2 * M - k < bins) emit(re, im, mg, 2 * M - k, cconj(X), false, inv_n, mag_is_re);
    }
    if (t == 0 && M < bins) {
      // Nyquist: X[M] = Re Z[0] - Im Z[0]
      emit(re, im, mg, M, make_float2(v[0].x - v[0].y, 0.f), true, inv_n, mag_is_re);
    }
  }
};

// ------------------------------------------------------------------ C2C IO
// Element n of a C2C line after the Cooley-Tukey pre-hook; at(m) fetches
// the line's raw element m (contiguous or strided lines).
template <class At>
__device__ __forceinline__ float2 c2c_pre_elem(const C2cArgs& a, const At& at, int n) {
  if (a.pre == 1) {  // eigen_fft.hpp:2493-2502
    float2 u = at(n);
    u.y = 0.f;
    return u;
  }
  if (a.pre == 2) {  // eigen_fft.hpp:2505-2531
    int m = n;
    bool cj = false;
    if (m > (a.N >> 1)) { m = a.N - m; cj = true; }
    float2 u = at(m);
    if (a.polar_in) u = polar_to_complex(u);
    if (m == 0 || m == (a.N >> 1)) u.y = 0.f;
    return cj ? cconj(u) : u;
  }
  return at(n);
}

struct C2cIO {
  C2cArgs a;

  __device__ __forceinline__ float2 elem(const float2* col, int n) const {
    return c2c_pre_elem(a, [col](int m) { return col[m]; }, n);
  }

  __device__ __forceinline__ float2 elem4(long long b, long long n) const {
    if (b >= a.batch) return make_float2(0.f, 0.f);
    const float2 u = elem(a.in + b * (long long)a.N, (int)n);
    return a.inverse ? cconj(u) : u;
  }
  __device__ __forceinline__ void emit4(long long b, long long k, float2 X) const {
    if (b >= a.batch) return;
    if (a.inverse) X = cscale(cconj(X), 1.0f / (float)a.N);
    a.out[b * (long long)a.N + k] = post_hook(X, (int)k, a.N, a.pf);
  }

  template <class S>
  __device__ __forceinline__ void load(long long b, int t, float2 (&v)[S::R], float2*, const Twiddles&) const {
    if (b >= a.batch) {
#pragma unroll
      for (int i = 0; i < S::R; ++i) v[i] = make_float2(0.f, 0.f);
      return;
    }
    const float2* col = a.in + b * (long long)a.N;
    // inverse = conj . forward . conj
    const float2 sg = make_float2(1.f, a.inverse ? -1.f : 1.f);
    if (a.pre == 0) {
#pragma unroll
      for (int i = 0; i < S::R; ++i) v[i] = __fmul2_rn(col[t + i * S::T], sg);
    } else {
#pragma unroll
      for (int i = 0; i < S::R; ++i) v[i] = __fmul2_rn(elem(col, t + i * S::T), sg);
    }
  }

  template <class S>
  __device__ __forceinline__ void store(long long b, int t, float2 (&v)[S::R], float2*,
                                        const Twiddles&) const {
    if (b >= a.batch) return;
    float2* col = a.out + b * (long long)a.N;
    const float sc = a.inverse ? 1.0f / (float)a.N : 1.0f;
    const float2 sg = make_float2(sc, a.inverse ? -sc : sc);
    if (!any_post(a.pf)) {
#pragma unroll
      for (int i = 0; i < S::R; ++i) col[t + i * S::T] = __fmul2_rn(v[i], sg);
    } else {
#pragma unroll
      for (int i = 0; i < S::R; ++i) {
        const int k = t + i * S::T;
        col[k] = post_hook(__fmul2_rn(v[i], sg), k, a.N, a.pf);
      }
    }
  }
};

// ------------------------------------------------------------------ complex batch IO
struct CplxBatchIO {
  CplxBatchArgs a;

  __device__ __forceinline__ float2 base(long long f, int m) const {
    if (m >= a.bins) return make_float2(0.f, 0.f);
    const long long o = f * (long long)a.bins + m;
    return make_float2(__ldg(a.in_re + o), __ldg(a.in_im + o));
  }

  __device__ __forceinline__ float2 elem(long long f, int n) const {
    const int half = a.N >> 1;
    if (a.c2r_half) {
      // fft_cffi.cpp:1072-1093 then, for Cooley-Tukey, eigen_fft.hpp:2505-2531
      int m = n;
      bool cj = false;
      if (m > half) { m = a.N - m; cj = true; }
      float2 u = base(f, m);
      if (m == 0 || m == half) u.y = 0.f;
      if (a.ct_pre == 2) {
        if (a.polar_in) u = polar_to_complex(u);
        if (m == 0 || m == half) u.y = 0.f;
      }
      return cj ? cconj(u) : u;
    }
    float2 u = base(f, n);
    if (a.ct_pre == 1) u.y = 0.f;
    return u;
  }

  __device__ __forceinline__ float2 elem4(long long f, long long n) const {
    if (f >= a.frames) return make_float2(0.f, 0.f);
    const float2 u = elem(f, (int)n);
    return a.inverse ? cconj(u) : u;
  }
  __device__ __forceinline__ void emit4(long long f, long long k, float2 X) const {
    if (f >= a.frames) return;
    if (a.inverse) X = cscale(cconj(X), 1.0f / (float)a.N);
    X = post_hook(X, (int)k, a.N, a.pf);
    float s = X.x;
    if (a.synth) s *= __ldg(a.synth + k);
    a.out[f * (long long)a.N + k] = s;
  }

  template <class S>
  __device__ __forceinline__ void load(long long f, int t, float2 (&v)[S::R], float2*, const Twiddles&) const {
    const bool ok = f < a.frames;
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      float2 u = ok ? elem(f, t + i * S::T) : make_float2(0.f, 0.f);
      v[i] = a.inverse ? cconj(u) : u;
    }
  }

  template <class S>
  __device__ __forceinline__ void store(long long f, int t, float2 (&v)[S::R], float2*,
                                        const Twiddles&) const {
    if (f >= a.frames) return;
    float* o = a.out + f * (long long)a.N;
    const float scale = 1.0f / (float)a.N;
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int k = t + i * S::T;
      float2 X = v[i];
      if (a.inverse) X = cscale(cconj(X), scale);
      X = post_hook(X, k, a.N, a.pf);
      float s = X.x;  // fft_cffi.cpp:1148-1156
      if (a.synth) s *= __ldg(a.synth + k);
      o[k] = s;
    }
  }
};

// Hermitian (C2R + half spectrum) complex batch as an N/2-point transform.
// With X[0..M] (M = N/2) the half spectrum of a real x,
//   E[m] = (X[m] + conj X[M-m]) / 2,  O[m] = (X[m] - conj X[M-m]) e^{+2 pi i m/N} / 2
// are the spectra of x[2m] and x[2m+1], so z = IDFT_M(E + i O) gives
// x[2m] = Re z[m], x[2m+1] = Im z[m].  A forward context transforms the
// conjugate spectrum instead and scales by N.  Each bin is read and (for
// Cooley-Tukey polar input) converted once, through the shared tile.
struct C2rHalfIO {
  CplxBatchArgs a;
  int logN;

  // X[k] as the Hermitian rebuild sees it (fft_cffi.cpp:1073-1078, and the
  // Cooley-Tukey pre-hook's polar conversion eigen_fft.hpp:2511-2522),
  // conjugated for a forward context.
  __device__ __forceinline__ float2 bin_of(float2 u, bool edge, float cs) const {
    if (edge) u.y = 0.f;
    if (a.ct_pre == 2 && a.polar_in) {
      u = polar_to_complex(u);
      if (edge) u.y = 0.f;
    }
    u.y *= cs;
    return u;
  }

  template <class S>
  __device__ __forceinline__ void load(long long f, int t, float2 (&v)[S::R], float2* sm,
                                       const Twiddles& tw) const {
    constexpr int M = S::M, T = S::T, R = S::R;
    constexpr int LN = S::LOGM + 1;
    const bool ok = f < a.frames;
    float2 xk[R];
    if (ok) {
      const float* re = a.in_re + f * (long long)a.bins;
      const float* im = a.in_im + f * (long long)a.bins;
      const float cs = a.inverse ? 1.f : -1.f;  // forward: conjugate spectrum
      // every load of the frame first (in flight together), then the
      // conversions and the tile writes
#pragma unroll
      for (int i = 0; i < R; ++i) xk[i] = make_float2(__ldg(re + t + i * T), __ldg(im + t + i * T));
      float2 xn = make_float2(0.f, 0.f);
      if (t == 0) xn = make_float2(__ldg(re + M), __ldg(im + M));
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int k = t + i * T;
        xk[i] = bin_of(xk[i], k == 0, cs);
        sm[pidx(k)] = xk[i];
      }
      if (t == 0) sm[pidx(M)] = bin_of(xn, true, cs);
    }
    GroupSync::sync<S>();
    const UntangleTw<S> w(tw, t);
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int m = t + i * T;
      float2 z = make_float2(0.f, 0.f);
      if (ok) {
        // conj of E + i O, E = (xk + conj xm) / 2, O = (xk - conj xm) conj(w) / 2:
        // A = xk + conj xm, B = xk - conj xm, Q = B conj(h), h = w / 2,
        // conj(A / 2 + i Q) = (A.x / 2 - Q.y, -(A.y / 2 + Q.x))
        const float2 xm = sm[pidx(M - m)];
        const float2 A = __ffma2_rn(xm, make_float2(1.f, -1.f), xk[i]);
        const float2 B = __ffma2_rn(xm, make_float2(-1.f, 1.f), xk[i]);
        const float2 h = w.half(i);
        const float2 Q = make_float2(__fmaf_rn(B.x, h.x, __fmul_rn(B.y, h.y)),
                                     __fmaf_rn(B.y, h.x, -__fmul_rn(B.x, h.y)));
        z = __ffma2_rn(A, make_float2(0.5f, -0.5f), make_float2(-Q.y, -Q.x));
      }
      v[i] = z;  // IDFT via conj . DFT . conj: the input already conjugated
    }
    GroupSync::sync<S>();  // the engine reuses the tile
  }

  template <class S>
  __device__ __forceinline__ void store(long long f, int t, float2 (&v)[S::R], float2*,
                                        const Twiddles&) const {
    if (f >= a.frames) return;
    constexpr int M = S::M;
    const float scale = a.inverse ? 1.0f / (float)M : 2.0f;  // forward: N/M
    const bool absval = a.pf.polar || a.pf.reduce;           // post hook on a real value
    float* o = a.out + f * (long long)a.N;
    const bool vec = aligned8(o) && (!a.synth || aligned8(a.synth));
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int m = t + i * S::T;
      float x0 = v[i].x * scale, x1 = -v[i].y * scale;
      if (absval) { x0 = fabsf(x0); x1 = fabsf(x1); }
      if (vec) {
        float2 s = make_float2(x0, x1);
        if (a.synth) s = __fmul2_rn(s, __ldg(reinterpret_cast<const float2*>(a.synth) + m));
        reinterpret_cast<float2*>(o)[m] = s;
      } else {
        if (a.synth) { x0 *= __ldg(a.synth + 2 * m); x1 *= __ldg(a.synth + 2 * m + 1); }
        o[2 * m] = x0;
        o[2 * m + 1] = x1;
      }
    }
  }
};

}  // namespace ffb
