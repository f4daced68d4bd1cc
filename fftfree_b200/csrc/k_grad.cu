// k_grad.cu -- gradient of the magnitude STFT with respect to the signals
// (the adjoint of the forward R2C half-spectrum STFT followed by |.|).
//
// For one frame s[n] = x[f*H + n] * w[n] (zero from the frame's sample
// count on) with half spectrum X[k], k = 0..N/2, and upstream gradient
// g[k] = dL/d|X[k]|:
//   dL/ds[n] = Re sum_{k=0}^{N/2} V[k] e^{+2 pi i k n / N},  V[k] = g[k] X[k] / |X[k]|
// (V = 0 where |X| = 0), i.e. the unnormalised Hermitian inverse of the
// half spectrum Y with Y[k] = V[k] for 0 < k < N/2 and Y[0] = 2 Re V[0],
// Y[N/2] = 2 Re V[N/2], halved -- computed as one N/2-point complex
// transform.  dL/dx[t] = sum over the frames f covering t of
// w[t - f*H] * dL/ds_f[t - f*H].
//
// The spectrum comes from the unit phasor X / |X| the forward pass saved, or
// is recomputed from x (long signals).  Two forms of the overlap-add
// adjoint, both gathers in frame order (deterministic, no atomics): the
// sliding form (hops N / 2^q) walks a run of frames per thread group and
// sums in a register window; the general form gives each block `span`
// consecutive samples of one signal, transforms every frame that touches
// them (a few frames of halo per block are transformed by both neighbours)
// and sums through a shared-memory accumulator.
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "fft_launch.cuh"

namespace ffb {
namespace {

template <class S>
struct SchedTag {
  using type = S;
};

template <int LOGM, class F>
cudaError_t with_r(int logr, F&& f) {
  switch (logr) {
    case 2: return f(SchedTag<Sched<LOGM, 2>>{});
    case 3: return f(SchedTag<Sched<LOGM, 3>>{});
    case 5:
      if constexpr (LOGM >= 9) return f(SchedTag<Sched<LOGM, 5>>{});
      else return f(SchedTag<Sched<LOGM, 4>>{});
    default: return f(SchedTag<Sched<LOGM, 4>>{});
  }
}

template <class F>
cudaError_t with_sched(int logm, int logr, F&& f) {
  switch (logm) {
    case 0: return with_r<0>(logr, f);
    case 1: return with_r<1>(logr, f);
    case 2: return with_r<2>(logr, f);
    case 3: return with_r<3>(logr, f);
    case 4: return with_r<4>(logr, f);
    case 5: return with_r<5>(logr, f);
    case 6: return with_r<6>(logr, f);
    case 7: return with_r<7>(logr, f);
    case 8: return with_r<8>(logr, f);
    case 9: return with_r<9>(logr, f);
    case 10: return with_r<10>(logr, f);
    case 11: return with_r<11>(logr, f);
    case 12: return with_r<12>(logr, f);
    case 13: return with_r<13>(logr, f);
    default: return cudaErrorInvalidValue;
  }
}

// Frame f of one signal as M complex points z[m] = (s[2m], s[2m+1]).
template <class S>
__device__ __forceinline__ void grad_load(const MagGradArgs& a, const float* pcm, long long f, bool ok, int t,
                                          float2 (&v)[S::R], long long* cnt_out) {
  long long cnt = 0;
  const float* src = ok ? stft_frame(pcm, a.pcm_len, 0, 0, a.W, a.H, f, &cnt) : pcm;
  *cnt_out = cnt;
  if (!ok) {
#pragma unroll
    for (int i = 0; i < S::R; ++i) v[i] = make_float2(0.f, 0.f);
    return;
  }
  if (cnt == a.N && aligned8(src) && (!a.win || aligned8(a.win))) {
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
#pragma unroll
  for (int i = 0; i < S::R; ++i) {
    const int n = 2 * (t + i * S::T);
    float x0 = 0.f, x1 = 0.f;
    if (n < cnt) x0 = a.win ? __ldg(src + n) * __ldg(a.win + n) : __ldg(src + n);
    if (n + 1 < cnt) x1 = a.win ? __ldg(src + n + 1) * __ldg(a.win + n + 1) : __ldg(src + n + 1);
    v[i] = make_float2(x0, x1);
  }
}

// The upstream gradient's factor: a.factor, times the device scalar a.scale
// when set (a loss's upstream gradient, read here rather than on the host).
__device__ __forceinline__ float grad_scale(const MagGradArgs& a) {
  return a.scale ? a.factor * __ldg(a.scale) : a.factor;
}

// dL/dX scaled onto the Hermitian half spectrum: V = g X / |X|, 0 at |X| = 0.
__device__ __forceinline__ float2 mag_chain(float2 X, float g) {
  const float m = cabs_fast(X.x, X.y);
  if (!(m > 0.f)) return make_float2(0.f, 0.f);
  const float s = g / m;
  return make_float2(X.x * s, X.y * s);
}

// Blocks per SM the register budget is sized for: the kernel holds a frame
// and its gradient spectrum in registers; capping registers at 64 (radix 8)
// or 80 (radix 16) keeps enough warps resident to hide the load latency.
template <class S>
constexpr int grad_min_blocks() {
  constexpr int want = S::R <= 8 ? 4 : (S::R == 16 ? 3 : 1);
  constexpr int fit64 = 65536 / (Launch<S>::BLOCK * 64);  // blocks at 64 registers a thread
  return want < fit64 ? want : (fit64 > 1 ? fit64 : 1);
}

// Hermitian half spectrum y (bins t + i*T, the Nyquist bin in ynyq on
// thread 0; DC and Nyquist already doubled) to the windowed frame gradient:
// v[i] holds samples n = 2m, 2m+1 (m = t + i*T) of w[n] dL/ds[n], zero from
// `cnt` on.  RAW leaves the window and the count to the caller: v[i] =
// (dL/ds[2m], -dL/ds[2m+1]).  The tile must be free on entry; it is free on
// return.
template <class S, bool RAW = false>
__device__ __forceinline__ void grad_inverse(const MagGradArgs& a, const float2 (&y)[S::R], float2 ynyq,
                                             long long cnt, int t, float2* sm, const Twiddles& tw,
                                             float2 (&v)[S::R]) {
  constexpr int T = S::T, R = S::R, M = S::M;
  constexpr int LN = S::LOGM + 1;  // N = 2M
  const UntangleTw<S> w(tw, t);  // e^{-2 pi i m / N}, m = t + i*T
  tile_write_natural<S>(y, t, sm);
  if (t == 0) sm[pidx(M)] = ynyq;
  GroupSync::sync<S>();

  // Hermitian half spectrum Y -> z' with x[2m] = Re, x[2m+1] = Im of the
  // unnormalised inverse: E = (Y[m] + conj Y[M-m]) / 2,
  // O = (Y[m] - conj Y[M-m]) e^{+2 pi i m/N} / 2, z' = IDFT_M(E + i O),
  // the IDFT taken as conj . DFT . conj.
#pragma unroll
  for (int i = 0; i < R; ++i) {
    // conj(E + i O) with A = Y[m] + conj Y[M-m], B = Y[m] - conj Y[M-m],
    // Q = B conj(h), h = w / 2: (A.x / 2 - Q.y, -(A.y / 2 + Q.x))
    const int m = t + i * T;
    const float2 ym = sm[pidx(M - m)];
    const float2 A = __ffma2_rn(ym, make_float2(1.f, -1.f), y[i]);
    const float2 B = __ffma2_rn(ym, make_float2(-1.f, 1.f), y[i]);
    const float2 h = w.half(i);
    const float2 Q = make_float2(__fmaf_rn(B.x, h.x, __fmul_rn(B.y, h.y)), __fmaf_rn(B.y, h.x, -__fmul_rn(B.x, h.y)));
    v[i] = __ffma2_rn(A, make_float2(0.5f, -0.5f), make_float2(-Q.y, -Q.x));
  }
  GroupSync::sync<S>();  // the engine reuses the tile
  fft_engine<S, GroupSync>(v, t, sm, tw);
  if constexpr (!RAW) {
    // dL/ds[2m] = Re, dL/ds[2m+1] = -Im, times the window, zero past the frame's samples.
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int n = 2 * (t + i * T);
      float d0 = v[i].x, d1 = -v[i].y;
      if (a.win) {
        d0 *= __ldg(a.win + n);
        d1 *= __ldg(a.win + n + 1);
      }
      if (n >= cnt) d0 = 0.f;
      if (n + 1 >= cnt) d1 = 0.f;
      v[i] = make_float2(d0, d1);
    }
  }
}

// One frame's gradient dL/ds, windowed: on return v[i] holds the samples
// n = 2m, 2m + 1 (m = t + i*T) of w[n] dL/ds_f[n], zero from the frame's
// sample count on.  Every group barrier is inside; the tile is free on
// return (its last reads are behind a barrier).
template <class S, bool RAW = false>
__device__ __forceinline__ void frame_grad(const MagGradArgs& a, const float* pcm, const float* gsig, long long f,
                                           bool ok, int t, float2* sm, const Twiddles& tw, float2 (&v)[S::R]) {
  constexpr int T = S::T, R = S::R, M = S::M;
  constexpr int LN = S::LOGM + 1;  // N = 2M
  const UntangleTw<S> w(tw, t);  // e^{-2 pi i k / N}, k = t + i*T
  long long cnt;
  grad_load<S>(a, pcm, f, ok, t, v, &cnt);
  // upstream gradient of this frame's bins, fetched before the transform
  const float* gf = gsig + (ok ? f : 0) * (long long)(M + 1);
  const float sc = grad_scale(a);
  float gk[R];
#pragma unroll
  for (int i = 0; i < R; ++i) gk[i] = ok ? sc * __ldg(gf + t + i * T) : 0.f;
  fft_engine<S, GroupSync>(v, t, sm, tw);

  // Untangle Z (the M-point transform of z) into X[k], k = t + i*T, and
  // apply the magnitude chain rule bin by bin.
  tile_write_natural<S>(v, t, sm);
  GroupSync::sync<S>();
  float2 y[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int k = t + i * T;
    const float2 zm = sm[pidx((M - k) & (M - 1))];
    float2 X = untangle_bin(v[i], zm, w.half(i));
    if (i == 0 && t == 0) {
      X.y = 0.f;  // DC is real
      const float2 V = mag_chain(X, gk[0]);
      y[i] = make_float2(2.f * V.x, 0.f);
    } else {
      y[i] = mag_chain(X, gk[i]);
    }
  }
  float2 ynyq = make_float2(0.f, 0.f);
  if (t == 0) {  // Nyquist X[M] = Re Z[0] - Im Z[0]
    const float xn = v[0].x - v[0].y;
    const float gn = ok ? sc * __ldg(gf + M) : 0.f;
    ynyq = make_float2(2.f * mag_chain(make_float2(xn, 0.f), gn).x, 0.f);
  }
  GroupSync::sync<S>();  // every read of Z is done
  grad_inverse<S, RAW>(a, y, ynyq, cnt, t, sm, tw, v);
}

// The same from the unit phasor U = X / |X| the forward pass saved:
// V = g U -- no forward transform, no signal read.
template <class S, bool RAW = false>
__device__ __forceinline__ void frame_grad_phasor(const MagGradArgs& a, const float* gsig, const float2* usig,
                                                  long long f, bool ok, int t, float2* sm, const Twiddles& tw,
                                                  float2 (&v)[S::R]) {
  constexpr int T = S::T, R = S::R, M = S::M;
  long long cnt = 0;
  if (ok) {
    cnt = a.pcm_len - f * (long long)a.H;
    if (cnt > a.W) cnt = a.W;
  }
  const long long off = (ok ? f : 0) * (long long)(M + 1);
  const float sc = grad_scale(a);
  float2 y[R];
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int k = t + i * T;
    float2 V = make_float2(0.f, 0.f);
    if (ok) V = cscale(__ldg(usig + off + k), sc * __ldg(gsig + off + k));
    y[i] = (i == 0 && t == 0) ? make_float2(2.f * V.x, 0.f) : V;  // DC is real
  }
  float2 ynyq = make_float2(0.f, 0.f);
  if (t == 0 && ok) ynyq = make_float2(2.f * sc * __ldg(gsig + off + M) * __ldg(usig + off + M).x, 0.f);  // Nyquist
  grad_inverse<S, RAW>(a, y, ynyq, cnt, t, sm, tw, v);
}

template <class S, bool PH, bool RAW = false>
__device__ __forceinline__ void frame_grad_any(const MagGradArgs& a, const float* pcm, const float2* psig,
                                               const float* gsig, long long f, bool ok, int t, float2* sm,
                                               const Twiddles& tw, float2 (&v)[S::R]) {
  if constexpr (PH) frame_grad_phasor<S, RAW>(a, gsig, psig, f, ok, t, sm, tw, v);
  else frame_grad<S, RAW>(a, pcm, gsig, f, ok, t, sm, tw, v);
}

// General form: each block owns `span` samples of one signal and gathers
// the frames that touch them through a shared-memory accumulator.
template <class S, bool PH>
__global__ void __launch_bounds__(Launch<S>::BLOCK, grad_min_blocks<S>()) k_stft_mag_grad(MagGradArgs a,
                                                                                          Twiddles tw) {
  extern __shared__ float2 smem[];
  constexpr int T = S::T, R = S::R, M = S::M;
  constexpr int G = Launch<S>::G, B = Launch<S>::BLOCK;
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  float2* sm = smem + g * S::SMEM;
  float* acc = reinterpret_cast<float*>(smem + G * S::SMEM);

  const long long per_sig = (a.pcm_len + a.span - 1) / a.span;
  const long long sig = blockIdx.x / per_sig;
  const long long s0 = (blockIdx.x - sig * per_sig) * (long long)a.span;
  const long long s1 = (s0 + a.span < a.pcm_len) ? s0 + a.span : a.pcm_len;
  const int ns = (int)(s1 - s0);
  for (int p = threadIdx.x; p < ns; p += B) acc[p] = 0.f;

  // frames f with f*H < s1 and f*H + W > s0 (fewer samples only at the end)
  const long long f_lo = (s0 >= a.W) ? (s0 - a.W) / a.H + 1 : 0;
  long long f_hi = (s1 - 1) / a.H;
  if (f_hi > a.frames - 1) f_hi = a.frames - 1;
  const float* pcm = PH ? nullptr : a.pcm + sig * a.sig_stride;
  const float* gsig = a.grad_mag + sig * a.frames * (long long)(M + 1);
  const float2* psig = PH ? a.phasor + sig * a.frames * (long long)(M + 1) : nullptr;
  __syncthreads();

  for (long long f0 = f_lo; f0 <= f_hi; f0 += G) {  // block-uniform loop
    const long long f = f0 + g;
    float2 v[R];
    frame_grad_any<S, PH>(a, pcm, psig, gsig, f, f <= f_hi, t, sm, tw, v);
    tile_write_natural<S>(v, t, sm);
    __syncthreads();  // every group's frame is in its tile

    // Overlap-add adjoint: each owned sample gathers this round's frames in
    // frame order.
    const long long last = (f0 + G - 1 < f_hi) ? f0 + G - 1 : f_hi;
    long long lo = f0 * (long long)a.H, hi = last * (long long)a.H + a.N;
    if (lo < s0) lo = s0;
    if (hi > s1) hi = s1;
    const int g_last = (int)(last - f0);
    for (long long p = lo + threadIdx.x; p < hi; p += B) {
      // frames f0 + gg with 0 <= p - (f0 + gg) * H < N
      const long long r = p - f0 * (long long)a.H;
      int gg = (r >= a.N) ? (int)((r - a.N) / a.H) + 1 : 0;
      int ge = (int)(r / a.H);
      if (ge > g_last) ge = g_last;
      float sum = acc[p - s0];
      for (; gg <= ge; ++gg) {
        const int n = (int)(r - (long long)gg * a.H);
        const float* tile = reinterpret_cast<const float*>(smem + gg * S::SMEM);
        sum += tile[2 * pidx(n >> 1) + (n & 1)];
      }
      acc[p - s0] = sum;
    }
    __syncthreads();  // tiles are reused by the next round
  }

  float* out = a.grad_pcm + sig * a.sig_stride + s0;
  for (int p = threadIdx.x; p < ns; p += B) out[p] = acc[p];
}

// Sliding form, for hops H = N / 2^QL with H a multiple of 2T: thread t
// holds samples 2(t + i*T) + {0, 1} of every frame, so the overlap-add
// partners of a sample in consecutive frames sit in the same thread,
// SH = H / 2T register slots apart.  Each group of T threads walks a run of
// `run` consecutive frames of one signal (plus the frames before it that
// reach into it), adds every frame's gradient into a register window, and
// after each frame writes the SH slots no later frame touches.  Groups are
// independent: no block barrier, no accumulator in shared memory.  The
// sums are taken in frame order, as in the general form.
// The sliding form also keeps the register window: 3 blocks of 256 threads
// (85 registers) at radix 8, 2 (128 registers) at radix 16.
template <class S>
constexpr int slide_min_blocks() {
  constexpr int want = S::R <= 8 ? 3 : 2;
  constexpr int fit80 = 65536 / (Launch<S>::BLOCK * 80);  // blocks at 80 registers a thread
  return want < fit80 ? want : (fit80 > 1 ? fit80 : 1);
}

// Two samples p, p + 1 of the output (p even), as one 8-byte store where
// the row is 8-byte aligned and both are inside the signal.
__device__ __forceinline__ void store_pair(float* out, long long p, long long L, float x0, float x1, bool vec) {
  if (vec && p + 1 < L) {
    *reinterpret_cast<float2*>(out + p) = make_float2(x0, x1);
  } else {
    if (p < L) out[p] = x0;
    if (p + 1 < L) out[p + 1] = x1;
  }
}

// One frame into the register window at rotation ROT: slot i of the frame
// (samples 2(t + iT) + {0, 1} past its start) adds into acc[(i + ROT*SH) % R]
// as one FFMA2 with the window taps (w2: the block's copy in shared memory,
// or null for no window); v holds (dL/ds[2m], -dL/ds[2m+1]), so
// the window keeps the second sum negated.  The SH slots that are then
// complete (acc[ROT*SH ..]) are written when `store` and cleared for the
// frames to come.  Rotating the window instead of shifting it costs no
// register moves.
template <class S, int QL, int ROT>
__device__ __forceinline__ void slide_step(float2 (&acc)[S::R], const float2 (&v)[S::R], const float2* w2, int t,
                                           bool store, float* out, long long base, long long L, bool vec) {
  constexpr int T = S::T, R = S::R, SH = R >> QL;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const float2 w = w2 ? w2[t + i * T] : make_float2(1.f, 1.f);  // w2: shared memory
    acc[(i + ROT * SH) % R] = __ffma2_rn(v[i], w, acc[(i + ROT * SH) % R]);
  }
  if (store) {
#pragma unroll
    for (int j = 0; j < SH; ++j)
      store_pair(out, base + 2 * (t + j * T), L, acc[ROT * SH + j].x, -acc[ROT * SH + j].y, vec);
  }
#pragma unroll
  for (int j = 0; j < SH; ++j) acc[ROT * SH + j] = make_float2(0.f, 0.f);
}

template <class S, int QL, int ROT = 0>
__device__ __forceinline__ void slide_step_at(int rot, float2 (&acc)[S::R], const float2 (&v)[S::R],
                                              const float2* w2, int t, bool store, float* out, long long base,
                                              long long L, bool vec) {
  if constexpr (ROT < (1 << QL)) {
    if (rot == ROT) slide_step<S, QL, ROT>(acc, v, w2, t, store, out, base, L, vec);
    else slide_step_at<S, QL, ROT + 1>(rot, acc, v, w2, t, store, out, base, L, vec);
  }
}

// After the last frame: the slots still pending (relative slots 0 .. R-SH-1
// of the frame that would follow, at rotation ROT) go out.
template <class S, int QL, int ROT = 0>
__device__ __forceinline__ void slide_tail_at(int rot, const float2 (&acc)[S::R], int t, float* out, long long base,
                                              long long L, bool vec) {
  constexpr int T = S::T, R = S::R, SH = R >> QL;
  if constexpr (ROT < (1 << QL)) {
    if (rot == ROT) {
#pragma unroll
      for (int i = 0; i < R - SH; ++i)
        store_pair(out, base + 2 * (t + i * T), L, acc[(ROT * SH + i) % R].x, -acc[(ROT * SH + i) % R].y, vec);
    } else {
      slide_tail_at<S, QL, ROT + 1>(rot, acc, t, out, base, L, vec);
    }
  }
}

template <class S, int QL, bool PH>
__global__ void __launch_bounds__(Launch<S>::BLOCK, slide_min_blocks<S>()) k_stft_mag_grad_slide(MagGradArgs a,
                                                                                                 Twiddles tw) {
  extern __shared__ float2 smem[];
  constexpr int T = S::T, R = S::R, M = S::M, G = Launch<S>::G;
  constexpr int SH = R >> QL;  // register slots per hop
  static_assert(SH >= 1, "hop of at least 2T samples");
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  float2* sm = smem + g * S::SMEM;
  // the window taps, once per block in shared memory after the groups' tiles
  // (every group reads the same taps at the same slots for every frame)
  const float2* w2 = nullptr;
  if (a.win) {
    float* wsm = reinterpret_cast<float*>(smem + G * S::SMEM);
    for (int p = threadIdx.x; p < 2 * M; p += blockDim.x) wsm[p] = __ldg(a.win + p);
    __syncthreads();
    w2 = reinterpret_cast<const float2*>(wsm);
  }
  const long long runs = (a.frames + a.run - 1) / a.run;
  const long long job = (long long)blockIdx.x * G + g;
  if (job >= a.signals * runs) return;  // the whole group leaves; no block barrier follows
  const long long sig = job / runs;
  const long long f_own = (job - sig * runs) * a.run;
  const long long f_end = (f_own + a.run < a.frames) ? f_own + a.run : a.frames;
  const long long halo = (long long)(1 << QL) - 1;  // earlier frames reaching into f_own*H
  const long long f_start = (f_own > halo) ? f_own - halo : 0;
  const float* pcm = PH ? nullptr : a.pcm + sig * a.sig_stride;
  const float* gsig = a.grad_mag + sig * a.frames * (long long)(M + 1);
  const float2* psig = PH ? a.phasor + sig * a.frames * (long long)(M + 1) : nullptr;
  float* out = a.grad_pcm + sig * a.sig_stride;
  const long long L = a.pcm_len;
  const bool vec = aligned8(out);

  float2 acc[R];
#pragma unroll
  for (int i = 0; i < R; ++i) acc[i] = make_float2(0.f, 0.f);
  int rot = 0;
  for (long long f = f_start; f < f_end; ++f) {
    float2 v[R];
    frame_grad_any<S, PH, true>(a, pcm, psig, gsig, f, true, t, sm, tw, v);
    long long cnt = L - f * (long long)a.H;  // the frame's samples; zero padding from there on
    if (cnt > a.W) cnt = a.W;
    if (cnt < 2 * M) {
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int n = 2 * (t + i * T);
        if (n >= cnt) v[i].x = 0.f;
        if (n + 1 >= cnt) v[i].y = 0.f;
      }
    }
    slide_step_at<S, QL>(rot, acc, v, w2, t, f >= f_own, out, f * (long long)a.H, L, vec);
    rot = (rot + 1) & ((1 << QL) - 1);
  }
  if (f_end == a.frames) {
    // the last run also writes the tail of the last frame and zeros the
    // samples no frame covers
    const long long base = f_end * (long long)a.H;
    slide_tail_at<S, QL>(rot, acc, t, out, base, L, vec);
    for (long long p = base + 2LL * (R - SH) * T + t; p < L; p += T) out[p] = 0.f;
  }
}

}  // namespace

int max_mag_grad_log() { return 14; }

// Radix of the sliding form: FFTFREE_GRAD_LOGR overrides it (sweeps).
static int slide_logr(int logm) {
  static const int env = [] {
    const char* e = std::getenv("FFTFREE_GRAD_LOGR");
    return e ? std::atoi(e) : 0;
  }();
  if (env == 3 || env == 4) return env;
  return (logm == 10) ? 4 : 3;
}

// Frames per thread group when the caller leaves it open (run < 0): among
// runs of 16 .. 64 frames, the one with the least work per group slot, a
// group slot being one of the G groups of a block resident on an SM.  Each
// group also transforms the `halo` frames before its run, and all groups take
// equally long, so a launch costs about ceil(jobs / slots) * (run + halo)
// frame transforms per slot.  On 64 signals of 509 frames (H = N/4, 1184
// slots) that is a run of 29: 1152 groups in one wave, where runs of 32 would
// leave 40 SMs with one block instead of two.
static long long slide_run(const MagGradArgs& a, const void* fn, int block, size_t smem, int G, int halo) {
  if (a.run > 0) return a.run;
  // resident blocks of this kernel on this device, queried once
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t>, long long> resident;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 32;
  }
  long long blocks = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = resident.find({fn, dev, smem});
    if (it != resident.end()) {
      blocks = it->second;
    } else {
      int sms = 0, per_sm = 0;
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return 32;
      }
      blocks = resident[{fn, dev, smem}] = (long long)sms * per_sm;
    }
  }
  const long long slots = blocks * G;
  long long best = 32, best_cost = -1;
  for (long long run = 16; run <= 64; ++run) {
    const long long jobs = a.signals * ((a.frames + run - 1) / run);
    const long long cost = ((jobs + slots - 1) / slots) * (run + halo);
    if (best_cost < 0 || cost < best_cost) best = run, best_cost = cost;
  }
  return best;
}

template <class S, int QL, bool PH>
static cudaError_t launch_slide(const MagGradArgs& a0, cudaStream_t st, uint64_t* launches) {
  using L = Launch<S>;
  // the groups' tiles, then the window taps
  const size_t smem = (size_t)L::G * S::SMEM * sizeof(float2) + (a0.win ? (size_t)a0.N * sizeof(float) : 0);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_stft_mag_grad_slide<S, QL, PH>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  MagGradArgs a = a0;
  a.run = (int)slide_run(a0, (const void*)k_stft_mag_grad_slide<S, QL, PH>, L::BLOCK, smem, L::G, (1 << QL) - 1);
  const long long jobs = a.signals * ((a.frames + a.run - 1) / a.run);
  const long long grid = (jobs + L::G - 1) / L::G;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
  Twiddles tw{twiddle_pyramid(0, st), twiddle_pass_tables(st)};
  k_stft_mag_grad_slide<S, QL, PH><<<(unsigned)grid, L::BLOCK, smem, st>>>(a, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

cudaError_t launch_stft_mag_grad(const MagGradArgs& a, int req_logr, cudaStream_t st, uint64_t* launches) {
  if (a.N < 2 || (a.N & (a.N - 1)) || a.signals <= 0 || a.pcm_len <= 0 || a.frames <= 0 || a.span <= 0 ||
      a.H <= 0 || a.W <= 0 || a.W > a.N)
    return cudaErrorInvalidValue;
  const int logm = ilog2i(a.N) - 1;
  if (logm + 1 > max_mag_grad_log()) return cudaErrorInvalidValue;

  // Sliding form when the hop is N / 2^q (q <= 3) and a multiple of 2T
  // (and the window taps can be read in pairs).
  if (a.run != 0 && logm >= 6 && (a.N % a.H) == 0 && (reinterpret_cast<uintptr_t>(a.win) & 7) == 0) {
    const int q = ilog2i(a.N / a.H);
    const int lr = slide_logr(logm);
    const int T = 1 << (logm - lr);
    if ((1 << q) == a.N / a.H && q <= 3 && (a.H % (2 * T)) == 0) {
      return with_sched(logm, lr, [&](auto tag) -> cudaError_t {
        using S = typename decltype(tag)::type;
        if constexpr (S::LOGM < 6 || (S::LOGR != 3 && S::LOGR != 4) || S::T > 1024) {
          return cudaErrorInvalidValue;
        } else {
          if (a.phasor) {
            switch (q) {
              case 0: return launch_slide<S, 0, true>(a, st, launches);
              case 1: return launch_slide<S, 1, true>(a, st, launches);
              case 2: return launch_slide<S, 2, true>(a, st, launches);
              default: return launch_slide<S, 3, true>(a, st, launches);
            }
          }
          switch (q) {
            case 0: return launch_slide<S, 0, false>(a, st, launches);
            case 1: return launch_slide<S, 1, false>(a, st, launches);
            case 2: return launch_slide<S, 2, false>(a, st, launches);
            default: return launch_slide<S, 3, false>(a, st, launches);
          }
        }
      });
    }
  }

  const int logr = choose_logr(logm, req_logr, true);
  if (logr < 0) return cudaErrorInvalidValue;
  return with_sched(logm, logr, [&](auto tag) -> cudaError_t {
    using S = typename decltype(tag)::type;
    if constexpr (S::T > 1024) {
      return cudaErrorInvalidValue;
    } else {
      using L = Launch<S>;
      const size_t smem = (size_t)L::G * S::SMEM * sizeof(float2) + (size_t)a.span * sizeof(float);
      if (smem > 227 * 1024) return cudaErrorInvalidValue;
      const void* fn = a.phasor ? (const void*)k_stft_mag_grad<S, true> : (const void*)k_stft_mag_grad<S, false>;
      if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
      }
      const long long per_sig = (a.pcm_len + a.span - 1) / a.span;
      const long long grid = per_sig * a.signals;
      if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
      Twiddles tw{twiddle_pyramid(0, st), twiddle_pass_tables(st)};
      if (a.phasor) k_stft_mag_grad<S, true><<<(unsigned)grid, L::BLOCK, smem, st>>>(a, tw);
      else k_stft_mag_grad<S, false><<<(unsigned)grid, L::BLOCK, smem, st>>>(a, tw);
      if (launches) ++*launches;
      return cudaGetLastError();
    }
  });
}

}  // namespace ffb
