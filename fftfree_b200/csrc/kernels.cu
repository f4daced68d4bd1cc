// kernels.cu -- single-pass batched FFT kernels for sm_100a and their
// launchers: real-frame STFT (fused framing, window, zero-pad, mirror, R2C
// half-size untangle, hooks, planar epilogue), complex C2C with the plan's
// hooks, complex/inverse batch, and the overlap-add gather.
#include "kernels.h"
#include "fft_engine.cuh"

#include <cmath>
#include <mutex>
#include <vector>

namespace ffb {

// ------------------------------------------------------------------ hooks
__device__ __forceinline__ float2 post_hook(float2 X, int k, int N, const PostFlags& pf) {
  // eigen_fft.hpp:2544-2595.  Polar/reduce apply below `upper`; above it the
  // R2C half branch has already zeroed the value, and (0,0) is a fixed point
  // of both, so applying them everywhere is equivalent.
  if (pf.r2c_half) {
    if (k > (N >> 1)) X = make_float2(0.f, 0.f);
    else if (k == 0 || k == (N >> 1)) X.y = 0.f;
  }
  if (pf.polar) {
    const float m = hypotf(X.x, X.y);
    const float ph = atan2f(X.y, X.x);
    X = make_float2(m, ph);
  } else if (pf.reduce) {
    X = make_float2(hypotf(X.x, X.y), 0.f);
  } else if (pf.clear_imag) {
    X.y = 0.f;
  }
  return X;
}

__device__ __forceinline__ float2 polar_to_complex(float2 u) {
  float s, c;
  sincosf(u.y, &s, &c);
  return make_float2(u.x * c, u.x * s);
}

// ------------------------------------------------------------------ STFT IO
struct StftIO {
  StftArgs a;
  int logN;

  __device__ __forceinline__ float sample(long long f, int n) const {
    // fft_cffi.cpp:765-791 framing (+ Cooley-Tukey C2R half mirror of the
    // pre-hook, eigen_fft.hpp:2523-2528, which on real frames is x[N-n]=x[n]).
    if (a.mirror && n > (a.N >> 1)) n = a.N - n;
    const long long start = f * (long long)a.H;
    long long cnt = a.pcm_len - start;
    if (cnt > a.W) cnt = a.W;
    if ((long long)n >= cnt) return 0.f;
    const float s = __ldg(a.pcm + start + n);
    return a.win ? s * __ldg(a.win + n) : s;
  }

  template <class S>
  __device__ __forceinline__ void load(long long f, int t, float2 (&v)[S::R], const Twiddles&) const {
    const bool ok = f < a.frames;
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int m = t + i * S::T;
      if (!ok) { v[i] = make_float2(0.f, 0.f); continue; }
      if (a.N == 1) v[i] = make_float2(sample(f, 0), 0.f);
      else v[i] = make_float2(sample(f, 2 * m), sample(f, 2 * m + 1));
    }
  }

  template <class S>
  __device__ __forceinline__ void store(long long f, int t, float2 (&v)[S::R], float2* sm,
                                        const Twiddles& tw) const {
    constexpr int M = S::M;
#pragma unroll
    for (int i = 0; i < S::R; ++i) sm[sw(t + i * S::T)] = v[i];
    __syncthreads();
    if (f >= a.frames) return;
    const int N = a.N;
    const long long ob = f * a.out_stride;
    for (int k = t; k < a.out_bins; k += S::T) {
      int kk = k;
      bool cj = false;
      if (kk > (N >> 1)) { kk = N - kk; cj = true; }
      float2 X;
      if (N == 1) {
        X = sm[0];
      } else {
        // Real-input untangle of the N/2-point transform Z of z[m] = x[2m] + i x[2m+1]:
        // X[k] = E + w^k O,  E = (Z[k] + conj Z[M-k]) / 2,  O = -i (Z[k] - conj Z[M-k]) / 2
        const float2 zk = sm[sw(kk & (M - 1))];
        const float2 zm = sm[sw((M - kk) & (M - 1))];
        const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 D = make_float2(zk.x - zm.x, zk.y + zm.y);
        const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
        X = cadd(E, cmul(tw_get(tw, logN, (unsigned)kk), O));
      }
      if (cj) X = cconj(X);
      if (a.inverse) X = cscale(cconj(X), 1.0f / (float)N);
      // Real input: DC and Nyquist are exactly real (imag +0), as in the
      // reference's radix-2 executors.
      if (kk == 0 || 2 * kk == N) X.y = 0.f;
      X = post_hook(X, k, N, a.pf);
      a.out_re[ob + k] = X.x;
      a.out_im[ob + k] = X.y;
      a.out_mag[ob + k] = (a.mag_from_real && a.pf.polar) ? X.x : hypotf(X.x, X.y);
    }
  }
};

// ------------------------------------------------------------------ C2C IO
struct C2cIO {
  C2cArgs a;

  __device__ __forceinline__ float2 elem(long long b, int n) const {
    const float2* col = a.in + b * (long long)a.N;
    if (a.pre == 1) {  // eigen_fft.hpp:2493-2502
      float2 u = col[n];
      u.y = 0.f;
      return u;
    }
    if (a.pre == 2) {  // eigen_fft.hpp:2505-2531
      int m = n;
      bool cj = false;
      if (m > (a.N >> 1)) { m = a.N - m; cj = true; }
      float2 u = col[m];
      if (a.polar_in) u = polar_to_complex(u);
      if (m == 0 || m == (a.N >> 1)) u.y = 0.f;
      return cj ? cconj(u) : u;
    }
    return col[n];
  }

  template <class S>
  __device__ __forceinline__ void load(long long b, int t, float2 (&v)[S::R], const Twiddles&) const {
    const bool ok = b < a.batch;
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      float2 u = ok ? elem(b, t + i * S::T) : make_float2(0.f, 0.f);
      v[i] = a.inverse ? cconj(u) : u;  // inverse = conj . forward . conj
    }
  }

  template <class S>
  __device__ __forceinline__ void store(long long b, int t, float2 (&v)[S::R], float2*,
                                        const Twiddles&) const {
    if (b >= a.batch) return;
    float2* col = a.out + b * (long long)a.N;
    const float scale = 1.0f / (float)a.N;
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int k = t + i * S::T;
      float2 X = v[i];
      if (a.inverse) X = cscale(cconj(X), scale);
      col[k] = post_hook(X, k, a.N, a.pf);
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

  template <class S>
  __device__ __forceinline__ void load(long long f, int t, float2 (&v)[S::R], const Twiddles&) const {
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

// ------------------------------------------------------------------ kernel
template <class S>
struct Launch {
  static constexpr int G = (S::T >= 256) ? 1 : 256 / S::T;  // transforms per block
  static constexpr int BLOCK = S::T * G;
};

template <class S, class IO>
__global__ void __launch_bounds__(Launch<S>::BLOCK)
k_fft(IO io, Twiddles tw) {
  extern __shared__ float2 smem[];
  constexpr int T = S::T;
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  const long long b = (long long)blockIdx.x * Launch<S>::G + g;
  float2* sm = smem + g * S::M;
  float2 v[S::R];
  io.template load<S>(b, t, v, tw);
  fft_engine<S>(v, t, sm, tw);
  io.template store<S>(b, t, v, sm, tw);
}

template <class S, class IO>
static cudaError_t run(const IO& io, long long nbatch, cudaStream_t st, uint64_t* launches) {
  using L = Launch<S>;
  if (nbatch <= 0) return cudaSuccess;
  const long long grid = (nbatch + L::G - 1) / L::G;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
  const size_t smem = (size_t)L::G * S::M * sizeof(float2);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_fft<S, IO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  Twiddles tw{twiddle_pyramid(0, st)};
  k_fft<S, IO><<<(unsigned)grid, L::BLOCK, smem, st>>>(io, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

// Compile-time table of instantiations: LOGM 0..13, LOGR 2..4 (clamped by
// Sched), threads per transform <= 1024.
template <class IO, int LOGM, int LOGR>
static cudaError_t run_if_valid(const IO& io, long long n, cudaStream_t st, uint64_t* l) {
  using S = Sched<LOGM, LOGR>;
  if constexpr (S::T > 1024) {
    return cudaErrorInvalidValue;
  } else {
    return run<S, IO>(io, n, st, l);
  }
}

template <class IO, int LOGM>
static cudaError_t dispatch_r(const IO& io, int logr, long long n, cudaStream_t st, uint64_t* l) {
  switch (logr) {
    case 2: return run_if_valid<IO, LOGM, 2>(io, n, st, l);
    case 3: return run_if_valid<IO, LOGM, 3>(io, n, st, l);
    default: return run_if_valid<IO, LOGM, 4>(io, n, st, l);
  }
}

template <class IO>
static cudaError_t dispatch(const IO& io, int logm, int logr, long long n, cudaStream_t st,
                            uint64_t* l) {
  switch (logm) {
    case 0: return dispatch_r<IO, 0>(io, logr, n, st, l);
    case 1: return dispatch_r<IO, 1>(io, logr, n, st, l);
    case 2: return dispatch_r<IO, 2>(io, logr, n, st, l);
    case 3: return dispatch_r<IO, 3>(io, logr, n, st, l);
    case 4: return dispatch_r<IO, 4>(io, logr, n, st, l);
    case 5: return dispatch_r<IO, 5>(io, logr, n, st, l);
    case 6: return dispatch_r<IO, 6>(io, logr, n, st, l);
    case 7: return dispatch_r<IO, 7>(io, logr, n, st, l);
    case 8: return dispatch_r<IO, 8>(io, logr, n, st, l);
    case 9: return dispatch_r<IO, 9>(io, logr, n, st, l);
    case 10: return dispatch_r<IO, 10>(io, logr, n, st, l);
    case 11: return dispatch_r<IO, 11>(io, logr, n, st, l);
    case 12: return dispatch_r<IO, 12>(io, logr, n, st, l);
    case 13: return dispatch_r<IO, 13>(io, logr, n, st, l);
    default: return cudaErrorInvalidValue;
  }
}

int max_single_pass_log() { return 13; }

int choose_logr(int logm, int requested_log) {
  if (logm > max_single_pass_log()) return -1;
  auto valid = [&](int lr) { return lr >= 2 && lr <= 4 && (logm - (lr < logm ? lr : logm)) <= 10; };
  if (requested_log >= 2 && requested_log <= 4 && valid(requested_log)) return requested_log;
  // default schedule: radix 16 for large transforms, 8 for mid, 4 for small
  int lr = (logm >= 10) ? 4 : (logm >= 6 ? 3 : 2);
  while (!valid(lr) && lr < 4) ++lr;
  return valid(lr) ? lr : -1;
}

static int ilog2i(long long n) {
  int l = 0;
  while ((1LL << l) < n) ++l;
  return l;
}

cudaError_t launch_stft(const StftArgs& a, int logr, cudaStream_t s, uint64_t* launches) {
  StftIO io{a, ilog2i(a.N)};
  const int logm = (a.N == 1) ? 0 : ilog2i(a.N) - 1;
  return dispatch(io, logm, logr, a.frames, s, launches);
}

cudaError_t launch_c2c(const C2cArgs& a, int logr, cudaStream_t s, uint64_t* launches) {
  C2cIO io{a};
  return dispatch(io, ilog2i(a.N), logr, a.batch, s, launches);
}

cudaError_t launch_cplx_batch(const CplxBatchArgs& a, int logr, cudaStream_t s, uint64_t* launches) {
  CplxBatchIO io{a};
  return dispatch(io, ilog2i(a.N), logr, a.frames, s, launches);
}

// ------------------------------------------------------------------ OLA
// fft_cffi.cpp:1119-1146: out[t] = sum over frames f with f*H <= t < f*H + N
// of frame_f[t - f*H], t < frames*N, accumulated in frame order; with COLA,
// divided by the summed weights where that sum exceeds 1e-12.
__global__ void k_ola(OlaArgs a) {
  const long long total = a.frames * (long long)a.N;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    long long fhi = t / a.H;
    if (fhi > a.frames - 1) fhi = a.frames - 1;
    const long long flo = (t >= a.N) ? (t - a.N) / a.H + 1 : 0;
    float acc = 0.f, nrm = 0.f;
    for (long long f = flo; f <= fhi; ++f) {
      const long long i = t - f * a.H;
      acc += __ldg(a.frames_buf + f * a.N + i);
      if (a.cola) nrm += a.weight ? __ldg(a.weight + i) : 1.0f;
    }
    if (a.cola && nrm > 1e-12f) acc /= nrm;
    a.out[t] = acc;
  }
}

cudaError_t launch_ola(const OlaArgs& a, cudaStream_t s, uint64_t* launches) {
  const long long total = a.frames * (long long)a.N;
  if (total <= 0) return cudaSuccess;
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_ola<<<(unsigned)blocks, 256, 0, s>>>(a);
  if (launches) ++*launches;
  return cudaGetLastError();
}

// ------------------------------------------------------------------ twiddles
namespace {
struct Pyramid {
  int max_log = -1;
  float2* dev = nullptr;
};
std::mutex g_tw_mu;
std::vector<Pyramid> g_tw;  // per device
}  // namespace

// exp(-2 pi i e / 2^L) in FP64 from the first octant with exact symmetry:
// quarter points are exactly 0 / +-1 and mirrored entries share bits.
static void octant_value(long long e, int L, double* c, double* s) {
  const long long n = 1LL << L;
  e &= (n - 1);
  if (L < 3) {
    // n in {1, 2, 4}: exact table
    static const double cs[4][2] = {{1, 0}, {0, -1}, {-1, 0}, {0, 1}};
    const long long q = (n == 1) ? 0 : e * (4 / n);
    *c = cs[q][0];
    *s = cs[q][1];
    return;
  }
  const long long n8 = n >> 3;
  const long long oct = e / n8;
  const long long r = e - oct * n8;
  // angle theta = 2 pi e / n = (pi/4) * oct + phi, phi = 2 pi r / n in [0, pi/4)
  auto base = [&](long long rr, double* cc, double* ss) {
    const double phi = 2.0 * M_PI * (double)rr / (double)n;
    *cc = std::cos(phi);
    *ss = std::sin(phi);
  };
  double cr, sr, cq, sq;
  base(r, &cr, &sr);          // cos/sin(phi)
  base(n8 - r, &cq, &sq);     // cos/sin(pi/4 - phi)
  double C, S;                // cos/sin(theta)
  switch (oct) {
    case 0: C = cr; S = sr; break;
    case 1: C = sq; S = cq; break;        // theta = pi/2 - (pi/4 - phi)
    case 2: C = -sr; S = cr; break;       // theta = pi/2 + phi
    case 3: C = -cq; S = sq; break;       // theta = pi - (pi/4 - phi)
    case 4: C = -cr; S = -sr; break;      // theta = pi + phi
    case 5: C = -sq; S = -cq; break;
    case 6: C = sr; S = -cr; break;       // theta = 3pi/2 + phi
    default: C = cq; S = -sq; break;      // theta = 2pi - (pi/4 - phi)
  }
  if (r == 0) {  // exact octant points
    const double h = std::sqrt(0.5);
    static const double ex[8][2] = {{1, 0}, {0, 0}, {0, 1}, {0, 0}, {-1, 0}, {0, 0}, {0, -1}, {0, 0}};
    if ((oct & 1) == 0) { C = ex[oct][0]; S = ex[oct][1]; }
    else {
      C = (oct == 1 || oct == 7) ? h : -h;
      S = (oct == 1 || oct == 3) ? h : -h;
    }
  }
  *c = C;
  *s = (S == 0.0) ? 0.0 : -S;  // exp(-i theta), without negative zeros
}

const float2* twiddle_pyramid(int max_log, cudaStream_t stream) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tw_mu);
  if ((int)g_tw.size() <= dev) g_tw.resize(dev + 1);
  Pyramid& p = g_tw[dev];
  const int want = max_log < 18 ? 18 : max_log;
  if (p.dev && p.max_log >= want) return p.dev;
  const size_t total = ((size_t)1 << (want + 1)) - 1;
  std::vector<float2> host(total);
  for (int L = 0; L <= want; ++L) {
    const size_t off = ((size_t)1 << L) - 1;
    for (long long e = 0; e < (1LL << L); ++e) {
      double c, s;
      octant_value(e, L, &c, &s);
      host[off + e] = make_float2((float)c, (float)s);
    }
  }
  float2* d = nullptr;
  if (cudaMalloc(&d, total * sizeof(float2)) != cudaSuccess) return p.dev;
  cudaMemcpyAsync(d, host.data(), total * sizeof(float2), cudaMemcpyHostToDevice, stream);
  cudaStreamSynchronize(stream);
  // The previous (smaller) table stays allocated: kernels still queued on
  // other streams may read it.
  p.dev = d;
  p.max_log = want;
  return p.dev;
}

}  // namespace ffb
