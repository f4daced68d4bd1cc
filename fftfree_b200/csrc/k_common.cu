// k_common.cu -- schedule choice, overlap-add gather and the twiddle tables.
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "fft_launch.cuh"

namespace ffb {

int max_single_pass_log() { return 13; }

// Radix 32 passes are instantiated for transforms of 2^9 points and up.
constexpr int kMinLogmRadix32 = 9;

static int env_logr(const char* name) {
  const char* e = std::getenv(name);
  return e ? std::atoi(e) : 0;
}

int choose_logr(int logm, int requested_log, bool real_path) {
  if (logm > max_single_pass_log()) return -1;
  auto valid = [&](int lr) {
    if (lr == 5) return logm >= kMinLogmRadix32 && logm - 5 <= 10;
    return lr >= 2 && lr <= 4 && (logm - (lr < logm ? lr : logm)) <= 10;
  };
  // FFTFREE_DEFAULT_LOGR_REAL / _COMPLEX override the default (sweeps)
  static const int env_real = env_logr("FFTFREE_DEFAULT_LOGR_REAL");
  static const int env_cplx = env_logr("FFTFREE_DEFAULT_LOGR_COMPLEX");
  const int env = real_path ? env_real : env_cplx;
  if (env >= 2 && env <= 5 && valid(env)) return env;
  // Default schedule, from B200 sweeps (one-warp transforms sync with warp
  // barriers, larger ones with a named barrier per transform): complex
  // transforms radix 32 at 1024 and 8192 points (a single exchange, or two
  // on 256 threads), radix 16 at 256..512 and 2048..4096, radix 8 below;
  // the real-input paths (an N/2-point transform plus the untangle) radix 16
  // at 512..2048 and 8192 complex points, radix 8 otherwise (2048 points:
  // R2C polar 0.0833 -> 0.0793 ms, C2R polar 0.0712 -> 0.0706 ms on 8192
  // frames of 4096 samples against radix 8).
  int lr;
  if (real_path) lr = (logm >= 9 && logm <= 11) || logm >= 13 ? 4 : (logm >= 6 ? 3 : 2);
  else if (logm == 10 || logm == 13) lr = 5;
  else lr = (logm >= 8) ? 4 : (logm >= 6 ? 3 : 2);
  // The plan's radix option / pattern (radix 4, 8 or 16; fft_cffi.hpp:67-72)
  // is a lower bound on the pass radix.  The reference's Stockham executor
  // runs radix-2 stages whatever it names (plan_support.hpp:136-150 only
  // selects an enum), so it fixes no result beyond rounding; a smaller
  // radix than the default only adds exchange passes on the GPU.
  if (requested_log >= 2 && requested_log <= 4 && requested_log > lr && valid(requested_log)) lr = requested_log;
  while (!valid(lr) && lr < 4) ++lr;
  return valid(lr) ? lr : -1;
}

// ------------------------------------------------------------------ OLA
// fft_cffi.cpp:1119-1146: out[t] = sum over frames f with f*H <= t < f*H + N
// of frame_f[t - f*H], t < frames*N, accumulated in frame order; with COLA,
// divided by the summed weights where that sum exceeds 1e-12.  Griffin-Lim
// asks for len = (frames-1)*H + N samples instead (phase_infer.hpp:147-168),
// which exceeds frames*N when H > N; samples no frame covers are 0.
__global__ void k_ola(OlaArgs a) {
  const long long total = a.len > 0 ? a.len : a.frames * (long long)a.N;
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

// The same sums four samples at a time with 16-byte accesses and 32-bit
// indexing, for N and H multiples of 4 (then the four samples t..t+3 lie in
// the same frames) and fewer than 2^31 samples in and out.
__global__ void k_ola4(OlaArgs a, int total4) {
  const int N = a.N, H = a.H, F = (int)a.frames;
  const float4* fb = reinterpret_cast<const float4*>(a.frames_buf);
  const float4* w4 = reinterpret_cast<const float4*>(a.weight);
  float4* out = reinterpret_cast<float4*>(a.out);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total4; q += gridDim.x * blockDim.x) {
    const int t = 4 * q;
    int fhi = t / H;
    if (fhi > F - 1) fhi = F - 1;
    const int flo = (t >= N) ? (t - N) / H + 1 : 0;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f), nrm = acc;
    for (int f = flo; f <= fhi; ++f) {
      const int i = t - f * H;
      const float4 v = __ldg(fb + (f * N + i) / 4);
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
      if (a.cola) {
        if (w4) {
          const float4 u = __ldg(w4 + i / 4);
          nrm.x += u.x;
          nrm.y += u.y;
          nrm.z += u.z;
          nrm.w += u.w;
        } else {
          nrm.x += 1.0f;
          nrm.y += 1.0f;
          nrm.z += 1.0f;
          nrm.w += 1.0f;
        }
      }
    }
    if (a.cola) {
      if (nrm.x > 1e-12f) acc.x /= nrm.x;
      if (nrm.y > 1e-12f) acc.y /= nrm.y;
      if (nrm.z > 1e-12f) acc.z /= nrm.z;
      if (nrm.w > 1e-12f) acc.w /= nrm.w;
    }
    out[q] = acc;
  }
}

cudaError_t launch_ola(const OlaArgs& a, cudaStream_t s, uint64_t* launches) {
  const long long total = a.len > 0 ? a.len : a.frames * (long long)a.N;
  if (total <= 0) return cudaSuccess;
  const auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if (a.N % 4 == 0 && a.H % 4 == 0 && total % 4 == 0 && total < (1LL << 31) &&
      a.frames * (long long)a.N < (1LL << 31) && al16(a.frames_buf) && al16(a.out) &&
      (!a.weight || al16(a.weight))) {
    const long long total4 = total / 4;
    long long blocks = (total4 + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_ola4<<<(unsigned)blocks, 256, 0, s>>>(a, (int)total4);
  } else {
    long long blocks = (total + 255) / 256;
    if (blocks > 148 * 64) blocks = 148 * 64;
    k_ola<<<(unsigned)blocks, 256, 0, s>>>(a);
  }
  if (launches) ++*launches;
  return cudaGetLastError();
}

// ------------------------------------------------------------------ Griffin-Lim
// phase_infer.hpp:190-207: out = |mag| e^{i arg(t)} per bin of the frames the
// forward pass produced; with a half spectrum, the DC bin's imaginary part
// and (even N) the Nyquist bin's are cleared.
__global__ void k_gl_project(const float* __restrict__ mag, const float* __restrict__ tr,
                             const float* __restrict__ ti, float* __restrict__ re, float* __restrict__ im,
                             long long nbins, int bins, int half, int even_n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbins;
       i += (long long)gridDim.x * blockDim.x) {
    const float ph = atan2f(__ldg(ti + i), __ldg(tr + i));
    const float m = __ldg(mag + i);
    float s, c;
    sincosf(ph, &s, &c);
    re[i] = m * c;
    float v = m * s;
    if (half) {
      const int k = (int)(i % bins);
      if (k == 0 || (even_n && bins > 1 && k == bins - 1)) v = 0.f;
    }
    im[i] = v;
  }
}

cudaError_t launch_gl_project(const float* mag, const float* tr, const float* ti, float* re, float* im,
                              long long nbins, int bins, int half, int even_n, cudaStream_t s) {
  if (nbins <= 0) return cudaSuccess;
  long long blocks = (nbins + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_gl_project<<<(unsigned)blocks, 256, 0, s>>>(mag, tr, ti, re, im, nbins, bins, half, even_n);
  return cudaGetLastError();
}

// phase_infer.hpp:133-137: out = magnitude * (cos, sin) of the initial phase,
// the float products of the reference.
__global__ void k_gl_init(const float* __restrict__ mag, const float2* __restrict__ cs, float* __restrict__ re,
                          float* __restrict__ im, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float m = __ldg(mag + i);
    const float2 u = __ldg(cs + i);
    re[i] = __fmul_rn(m, u.x);
    im[i] = __fmul_rn(m, u.y);
  }
}

cudaError_t launch_gl_init(const float* mag, const float2* cs, float* re, float* im, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_gl_init<<<(unsigned)blocks, 256, 0, s>>>(mag, cs, re, im, n);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ streaming ISTFT
__global__ void k_stream_ola(StreamOlaArgs a) {
  const long long total = a.count + (a.keep_carry ? a.N : 0);
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < total;
       j += (long long)gridDim.x * blockDim.x) {
    float acc = (j < a.N) ? a.carry[j] : 0.f;
    float nrm = (a.use_norm && j < a.N) ? a.carry_nrm[j] : 0.f;
    long long f0 = (j >= a.N) ? (j - a.N) / a.E + 1 : 0;
    long long f1 = j / a.E;
    if (f1 > a.F - 1) f1 = a.F - 1;
    for (long long f = f0; f <= f1; ++f) {
      const int i = (int)(j - f * a.E);
      acc += __ldg(a.frames + f * a.N + i);
      if (a.use_norm) nrm += a.weight ? __ldg(a.weight + i) : 1.0f;
    }
    if (j < a.count) {
      if (a.use_norm && fabsf(nrm) > 1e-12f) acc /= nrm;
      a.out[j] = acc;
    } else {
      a.new_carry[j - a.count] = acc;
      if (a.use_norm) a.new_nrm[j - a.count] = nrm;
    }
  }
}

cudaError_t launch_stream_ola(const StreamOlaArgs& a, cudaStream_t s) {
  const long long total = a.count + (a.keep_carry ? a.N : 0);
  if (total <= 0) return cudaSuccess;
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_stream_ola<<<(unsigned)blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ minimum phase
// fft_cffi.cpp:2104-2160 (phase_infer_execute, mode 1).  Log-amplitude
// spectrum: frame f, point k of N: log(max(eps, |X|)) with the half
// spectrum mirrored (points N-k from k, k < N/2), imaginary parts 0.
__global__ void k_minphase_log(const float* __restrict__ mag, float2* __restrict__ spec, long long frames, int N,
                               int bins, int half) {
  const long long total = frames * (long long)N;
  const float eps = 1e-20f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / N;
    const int k = (int)(i - f * N);
    int src = k;
    if (half) {
      // k <= N/2 from bin k; N-k (0 < k < N/2) mirrors bin k
      if (k > N / 2) src = N - k;
    }
    const float m = (src < bins) ? __ldg(mag + f * bins + src) : 0.f;
    spec[i] = make_float2(logf(fmaxf(eps, m)), 0.f);
  }
}

// Causal shaping of the real cepstrum: points 1 .. (N+1)/2 - 1 doubled,
// N/2 + 1 .. N-1 cleared (point 0 and, for even N, N/2 kept).
__global__ void k_minphase_fold(float2* __restrict__ cep, long long frames, int N) {
  const long long total = frames * (long long)N;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(i % N);
    if (n >= 1 && n < (N + 1) / 2) {
      const float2 c = cep[i];
      cep[i] = make_float2(2.0f * c.x, 2.0f * c.y);
    } else if (n >= N / 2 + 1) {
      cep[i] = make_float2(0.f, 0.f);
    }
  }
}

// Minimum-phase spectrum from the complex log spectrum L: exp(Re L) e^{i Im L},
// bins 0 .. bins-1 of every frame into planar re / im.
__global__ void k_minphase_exp(const float2* __restrict__ lg, float* __restrict__ re, float* __restrict__ im,
                               long long frames, int N, int bins) {
  const long long total = frames * (long long)bins;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / bins;
    const int k = (int)(i - f * bins);
    const float2 L = lg[f * N + k];
    const float a = expf(L.x);
    float s, c;
    sincosf(L.y, &s, &c);
    re[i] = a * c;
    im[i] = a * s;
  }
}

static unsigned elem_blocks(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)(b > 0 ? b : 1);
}

cudaError_t launch_minphase_log(const float* mag, float2* spec, long long frames, int N, int bins, int half,
                                cudaStream_t s) {
  if (frames <= 0 || N <= 0) return cudaSuccess;
  k_minphase_log<<<elem_blocks(frames * N), 256, 0, s>>>(mag, spec, frames, N, bins, half);
  return cudaGetLastError();
}

cudaError_t launch_minphase_fold(float2* cep, long long frames, int N, cudaStream_t s) {
  if (frames <= 0 || N <= 0) return cudaSuccess;
  k_minphase_fold<<<elem_blocks(frames * N), 256, 0, s>>>(cep, frames, N);
  return cudaGetLastError();
}

cudaError_t launch_minphase_exp(const float2* lg, float* re, float* im, long long frames, int N, int bins,
                                cudaStream_t s) {
  if (frames <= 0 || bins <= 0) return cudaSuccess;
  k_minphase_exp<<<elem_blocks(frames * bins), 256, 0, s>>>(lg, re, im, frames, N, bins);
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


namespace {
std::vector<float2*> g_pass;  // per device, guarded by g_tw_mu
}

// Per-pass twiddle tables (layout in fft_engine.cuh, pass_table_offset):
// w[(r-1)*Ns + k] = exp(-2 pi i k r / (Ns R)), built in FP64 with the same
// octant symmetry as the pyramid.
const float2* twiddle_pass_tables(cudaStream_t stream) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tw_mu);
  if ((int)g_pass.size() <= dev) g_pass.resize(dev + 1, nullptr);
  if (g_pass[dev]) return g_pass[dev];
  const long long total = pass_table_size();
  std::vector<float2> host((size_t)total);
  for (int lr = 1; lr <= 5; ++lr) {
    const int R = 1 << lr;
    for (int lns = 0; lns <= kPassMaxLog; ++lns) {
      const long long Ns = 1LL << lns;
      const long long off = pass_table_offset(lr, lns);
      for (int r = 1; r < R; ++r)
        for (long long k = 0; k < Ns; ++k) {
          double c, s;
          octant_value(k * r, lns + lr, &c, &s);
          host[(size_t)(off + (r - 1) * Ns + k)] = make_float2((float)c, (float)s);
        }
    }
  }
  float2* d = nullptr;
  if (cudaMalloc(&d, host.size() * sizeof(float2)) != cudaSuccess) return nullptr;
  cudaMemcpyAsync(d, host.data(), host.size() * sizeof(float2), cudaMemcpyHostToDevice, stream);
  cudaStreamSynchronize(stream);
  g_pass[dev] = d;
  return d;
}

}  // namespace ffb