// stream.cpp -- streaming STFT/ISTFT buffers, Griffin-Lim and phase
// inference: the reference's host-side drivers over the batched entry points
// (fft_cffi.cpp:1342-1742, 2058-2248; phase_infer.hpp).  Every transform they
// issue runs through the GPU entry points of abi.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../../include/fft_cffi.h"
#include "../../include/fftfree_b200.h"
#include "context.h"
#include "kernels.h"

namespace ffb {
namespace {

// fn(lo, hi) over [0, n) split into contiguous ranges, one per host thread
// (up to 16); small n on the calling thread alone.
template <class Fn>
void parallel_ranges(size_t n, Fn&& fn) {
  const size_t kMinPerThread = 1 << 15;
  size_t t = std::thread::hardware_concurrency();
  t = std::max<size_t>(1, std::min<size_t>({t, 16, n / kMinPerThread}));
  if (t <= 1) {
    fn(size_t(0), n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(t - 1);
  const size_t per = (n + t - 1) / t;
  for (size_t k = 1; k < t; ++k) {
    const size_t lo = std::min(n, k * per), hi = std::min(n, lo + per);
    pool.emplace_back([&fn, lo, hi] { fn(lo, hi); });
  }
  fn(size_t(0), std::min(n, per));
  for (std::thread& th : pool) th.join();
}

// Angle i of the n initial Griffin-Lim phases, as phase_infer.hpp:128-135
// draws them: std::uniform_real_distribution<float>(-pi, pi) over
// std::mt19937(seed), one 32-bit draw per angle (libstdc++'s
// generate_canonical<float, 24>: u = float(x) / 2^32, 1 - 2^-24 where that
// rounds to 1, then u * (b - a) + a in float).
inline float gl_angle(uint32_t x) {
  const float a = -3.14159265358979323846f, b = 3.14159265358979323846f;
  float u = (float)x / 4294967296.0f;
  if (u >= 1.0f) u = std::nextafter(1.0f, 0.0f);
  return u * (b - a) + a;
}

// MT19937 tempering of a state word (Matsumoto and Nishimura, 1998).
inline uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  return y ^ (y >> 18);
}

// The n initial phasors (cos, sin) of the angles above into the pinned host
// array out[], each block of them copied on to dev[] on stream s as soon as
// it is complete (std::cos / std::sin of the float angle).  The generator's
// state recurrence
//   x[k+624] = x[k+397] ^ (y >> 1) ^ (y odd ? 0x9908b0df : 0),
//   y = (x[k] & 0x80000000) | (x[k+1] & 0x7fffffff),
// with x[0..623] the standard seeding, runs sequentially over one array (x,
// kept by the caller between calls) on the calling thread; draw j is
// temper(x[624 + j]).  The tempering, the conversion, the cosines and sines
// and the copies of each block run on worker threads as the recurrence
// passes the block's end.  The first draws are checked against std::mt19937
// and std::uniform_real_distribution themselves; on a mismatch every angle
// comes from them.  Returns false if a copy could not be enqueued.
bool gl_initial_phasors(uint32_t seed, size_t n, std::vector<uint32_t>& x, float2* out, float2* dev,
                        int device, cudaStream_t s) {
  if (n == 0) return true;
  if (x.size() < n + 624) x.resize(n + 624);
  uint32_t* xs = x.data();
  xs[0] = seed;
  for (uint32_t i = 1; i < 624; ++i) xs[i] = 1812433253u * (xs[i - 1] ^ (xs[i - 1] >> 30)) + i;
  auto recur = [xs](size_t k0, size_t k1) {
    for (size_t k = k0; k < k1; ++k) {
      const uint32_t y = (xs[k] & 0x80000000u) | (xs[k + 1] & 0x7fffffffu);
      xs[k + 624] = xs[k + 397] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
  };
  const float kPi = 3.14159265358979323846f;
  const size_t check = std::min<size_t>(n, 2 * 624 + 16);
  recur(0, check);
  {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> dist(-kPi, kPi);
    bool same = true;
    for (size_t j = 0; j < check && same; ++j) same = dist(rng) == gl_angle(mt_temper(xs[624 + j]));
    if (!same) {
      std::mt19937 r2(seed);
      std::uniform_real_distribution<float> d2(-kPi, kPi);
      for (size_t j = 0; j < n; ++j) out[j].x = d2(r2);
      parallel_ranges(n, [&](size_t lo, size_t hi) {
        for (size_t j = lo; j < hi; ++j) {
          const float ang = out[j].x;
          out[j] = make_float2(std::cos(ang), std::sin(ang));
        }
      });
      return cudaMemcpyAsync(dev, out, n * sizeof(float2), cudaMemcpyHostToDevice, s) == cudaSuccess;
    }
  }
  const size_t kBlock = size_t(1) << 16;
  const size_t blocks = (n + kBlock - 1) / kBlock;
  std::atomic<size_t> produced{check}, next{0};
  std::atomic<bool> failed{false};
  auto work = [&](bool wait) {
    if (wait && cudaSetDevice(device) != cudaSuccess) failed = true;
    for (;;) {
      const size_t b = next.fetch_add(1);
      if (b >= blocks) return;
      const size_t lo = b * kBlock, hi = std::min(n, lo + kBlock);
      // the calling thread produces every block before it takes one
      while (wait && produced.load(std::memory_order_acquire) < hi) std::this_thread::yield();
      for (size_t j = lo; j < hi; ++j) {
        const float ang = gl_angle(mt_temper(xs[624 + j]));
        out[j] = make_float2(std::cos(ang), std::sin(ang));
      }
      if (cudaMemcpyAsync(dev + lo, out + lo, (hi - lo) * sizeof(float2), cudaMemcpyHostToDevice, s) !=
          cudaSuccess)
        failed = true;
    }
  };
  size_t t = std::thread::hardware_concurrency();
  t = std::max<size_t>(1, std::min<size_t>({t, 16, blocks}));
  std::vector<std::thread> pool;
  pool.reserve(t - 1);
  for (size_t k = 1; k < t; ++k) pool.emplace_back(work, true);
  for (size_t k = check; k < n; k += kBlock) {
    const size_t k1 = std::min(n, k + kBlock);
    recur(k, k1);
    produced.store(k1, std::memory_order_release);
  }
  work(false);
  for (std::thread& th : pool) th.join();
  return !failed;
}

bool verbose() {
  static const bool v = [] {
    const char* e = std::getenv("FFTFREE_VERBOSE");
    return e && *e && e[0] != '0';
  }();
  return v;
}

int stream_window(const FftContext* c) { return c->window > 0 ? c->window : c->N; }
int stream_hop(const FftContext* c) { return c->hop > 0 ? c->hop : stream_window(c); }

size_t stream_backlog(const FftContext* c) { return c->s_end > c->s_off ? c->s_end - c->s_off : 0; }

size_t stream_available_frames(const FftContext* c) {
  const size_t backlog = stream_backlog(c);
  const int W = stream_window(c), H = stream_hop(c);
  if (backlog < (size_t)W || W <= 0 || H <= 0) return 0;
  return 1 + (backlog - (size_t)W) / (size_t)H;
}

size_t stream_bins(const FftContext* c) {
  const size_t n = (size_t)std::max(c->N, 1);
  return c->half_spectrum ? n / 2 + 1 : n;
}

void check(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error("cuda");
}

bool on_device(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Room for `extra` more samples after [s_off, s_end): the backlog moves to
// the front of a (possibly larger) second buffer when the first is full.
float* stream_reserve(FftContext* c, size_t extra) {
  const size_t backlog = stream_backlog(c);
  const size_t cap = c->d_stream.cap / sizeof(float);
  if (c->d_stream.p && c->s_end + extra <= cap) return static_cast<float*>(c->d_stream.p);
  const size_t want = std::max<size_t>(2 * (backlog + extra), 1 << 16);
  float* dst = static_cast<float*>(c->d_stream2.get(want * sizeof(float)));
  if (backlog)
    check(cudaMemcpyAsync(dst, static_cast<float*>(c->d_stream.p) + c->s_off, backlog * sizeof(float),
                          cudaMemcpyDeviceToDevice, c->stream));
  std::swap(c->d_stream.p, c->d_stream2.p);
  std::swap(c->d_stream.cap, c->d_stream2.cap);
  c->s_off = 0;
  c->s_end = backlog;
  return dst;
}

size_t queue_pending(const FftContext* c) { return c->q_end > c->q_off ? c->q_end - c->q_off : 0; }

// Room for `extra` more emitted samples at the queue's tail.
float* queue_reserve(FftContext* c, size_t extra) {
  const size_t pending = queue_pending(c);
  const size_t cap = c->d_queue.cap / sizeof(float);
  if (c->d_queue.p && c->q_end + extra <= cap) return static_cast<float*>(c->d_queue.p);
  const size_t want = std::max<size_t>(2 * (pending + extra), 1 << 14);
  float* dst = static_cast<float*>(c->d_queue2.get(want * sizeof(float)));
  if (pending)
    check(cudaMemcpyAsync(dst, static_cast<float*>(c->d_queue.p) + c->q_off, pending * sizeof(float),
                          cudaMemcpyDeviceToDevice, c->stream));
  std::swap(c->d_queue.p, c->d_queue2.p);
  std::swap(c->d_queue.cap, c->d_queue2.cap);
  c->q_off = 0;
  c->q_end = pending;
  return dst;
}

// fft_cffi.cpp:1425-1447: up to max_samples (0: all) queued samples to out_pcm
size_t queue_emit(FftContext* c, float* out_pcm, size_t max_samples) {
  const size_t pending = queue_pending(c);
  if (pending == 0) return 0;
  size_t take = pending;
  if (max_samples != 0 && take > max_samples) take = max_samples;
  if (!out_pcm || take == 0) return 0;
  check(cudaMemcpyAsync(out_pcm, static_cast<float*>(c->d_queue.p) + c->q_off, take * sizeof(float),
                        cudaMemcpyDefault, c->stream));
  check(cudaStreamSynchronize(c->stream));
  c->q_off += take;
  if (c->q_off >= c->q_end) c->q_off = c->q_end = 0;
  return take;
}

// cola_window_weight (fft_cffi.cpp:210-226) on the device: analysis x
// synthesis taps with windows enabled, else nullptr (weight 1)
const float* stream_weight(FftContext* c) {
  if (!c->windows_enabled) return nullptr;
  const int n = std::max(c->N, 1);
  if (c->sweight_n != n) {
    std::vector<float> w(n);
    for (int i = 0; i < n; ++i) {
      const float a = (size_t)i < c->analysis_win.size() ? c->analysis_win[i] : 1.0f;
      const float s = (size_t)i < c->synthesis_win.size() ? c->synthesis_win[i] : 1.0f;
      w[i] = a * s;
    }
    float* d = static_cast<float*>(c->d_sweight.get(n * sizeof(float)));
    check(cudaMemcpyAsync(d, w.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    check(cudaStreamSynchronize(c->stream));
    c->sweight_n = n;
  }
  return static_cast<const float*>(c->d_sweight.p);
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" {

FFT_CFFI_API void fft_stream_reset(void* handle) {
  FftContext* c = as_ctx(handle);
  if (!c) return;
  c->s_off = c->s_end = 0;
  c->q_off = c->q_end = 0;
  c->acc_len = c->nrm_len = 0;
}

FFT_CFFI_API size_t fft_stream_pending_frames(void* handle) {
  FftContext* c = as_ctx(handle);
  return c ? stream_available_frames(c) : 0;
}

FFT_CFFI_API size_t fft_stream_backlog_samples(void* handle) {
  FftContext* c = as_ctx(handle);
  return c ? stream_backlog(c) : 0;
}

FFT_CFFI_API size_t fft_stream_pending_pcm(void* handle) {
  FftContext* c = as_ctx(handle);
  if (!c || !c->inverse) return 0;
  return queue_pending(c);
}

FFT_CFFI_API size_t fft_stream_push_pcm(void* handle, const float* pcm, size_t samples,
                                        float* out_real, float* out_imag, float* out_mag,
                                        size_t max_frames, int flush_mode) {
  // fft_cffi.cpp:1508-1595.  The backlog lives on the device: a push appends
  // the new samples (one copy) and the frames run straight from the backlog
  // -- the reference's host re-framing into a chunk gives the same samples
  // (frame f of the chunk is backlog[fH, fH + W)).  The reference prints a
  // diagnostic line on every call; here that needs FFTFREE_VERBOSE.
  (void)flush_mode;
  FftContext* c = as_ctx(handle);
  if (!c) {
    if (verbose()) std::fprintf(stderr, "[fft_stream_push_pcm] handle is NULL\n");
    return 0;
  }
  try {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
      int dev;
      ~Restore() {
        if (dev >= 0) cudaSetDevice(dev);
      }
    } restore{prev != c->device ? prev : -1};
    if (samples > 0 && pcm) {
      float* buf = stream_reserve(c, samples);
      check(cudaMemcpyAsync(buf + c->s_end, pcm, samples * sizeof(float), cudaMemcpyDefault, c->stream));
      // the caller may reuse its buffer on return (the reference copies it)
      if (!on_device(pcm)) check(cudaStreamSynchronize(c->stream));
      c->s_end += samples;
    }
    const int W = stream_window(c), H = stream_hop(c);
    if (verbose())
      std::fprintf(stderr, "[fft_stream_push_pcm] samples=%zu W=%d H=%d backlog=%zu\n", samples, W, H,
                   stream_backlog(c));
    if (W <= 0 || H <= 0) return 0;
    const size_t backlog = stream_backlog(c);
    const size_t available = stream_available_frames(c);
    if (available == 0) return 0;
    size_t frames = available;
    if (max_frames != 0 && frames > max_frames) frames = max_frames;
    size_t pcm_len = (size_t)W + (frames - 1) * (size_t)H;
    if (pcm_len > backlog) pcm_len = backlog;
    const size_t bins = stream_bins(c);
    const size_t ob = frames * bins * sizeof(float);
    float* rt = out_real ? out_real : static_cast<float*>(c->d_sre.get(ob));
    float* it = out_imag ? out_imag : static_cast<float*>(c->d_sim.get(ob));
    float* mt = out_mag ? out_mag : static_cast<float*>(c->d_smg.get(ob));
    const float* src = static_cast<const float*>(c->d_stream.p) + c->s_off;
    const size_t produced = fft_execute_batched(handle, src, pcm_len, rt, it, mt, 2, 0, frames);
    if (produced == 0) return 0;
    c->s_off += produced * (size_t)H;
    if (c->s_off >= c->s_end) c->s_off = c->s_end = 0;
    return produced;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API size_t fft_stream_push_spectrum(void* handle, const float* in_real,
                                             const float* in_imag, size_t frames, float* out_pcm,
                                             size_t max_samples, int flush_mode) {
  // fft_cffi.cpp:1597-1742 with the accumulator, the COLA norm and the queue
  // of emitted samples on the device: one inverse batch and one overlap-add
  // launch per push (k_stream_ola) in place of the per-frame host loop.
  FftContext* c = as_ctx(handle);
  if (!c || !c->inverse) return 0;
  try {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    struct Restore {
      int dev;
      ~Restore() {
        if (dev >= 0) cudaSetDevice(dev);
      }
    } restore{prev != c->device ? prev : -1};
    const size_t plan_n = (size_t)std::max(c->N, 1);
    const int N = (int)plan_n;
    const size_t nb = plan_n * sizeof(float);
    if (c->acc_len != plan_n) {
      check(cudaMemsetAsync(c->d_acc.get(nb), 0, nb, c->stream));
      c->acc_len = plan_n;
    }
    const bool use_norm = (c->cola_mode == FFT_COLA_NORMALIZE);
    if (use_norm) {
      if (c->nrm_len != plan_n) {
        check(cudaMemsetAsync(c->d_nrm.get(nb), 0, nb, c->stream));
        c->nrm_len = plan_n;
      }
    } else {
      c->nrm_len = 0;
    }
    const bool final_flush = (flush_mode == FFT_STREAM_FLUSH_FINAL);
    StreamOlaArgs o{};
    o.N = N;
    o.E = (int)std::min<size_t>((size_t)std::max(stream_hop(c), 1), plan_n);
    o.carry = static_cast<const float*>(c->d_acc.p);
    o.carry_nrm = use_norm ? static_cast<const float*>(c->d_nrm.p) : nullptr;
    o.weight = use_norm ? stream_weight(c) : nullptr;
    o.use_norm = use_norm ? 1 : 0;
    o.keep_carry = final_flush ? 0 : 1;
    bool run = false;
    if (frames > 0) {
      if (!in_real) return queue_emit(c, out_pcm, max_samples);
      // A NULL imaginary part fails the batch (as in the reference), which
      // then only drains what is queued.
      float* fr = static_cast<float*>(c->d_ifr.get(frames * plan_n * sizeof(float)));
      size_t produced = fft_execute_complex_batched(handle, in_real, in_imag, frames, fr, 2, 0, frames);
      if (produced == 0) return queue_emit(c, out_pcm, max_samples);
      if (produced > frames) produced = frames;
      o.frames = fr;
      o.F = (long long)produced;
      o.count = final_flush ? (long long)(produced - 1) * o.E + N : (long long)produced * o.E;
      run = true;
    } else if (final_flush) {
      // FINAL with no frames: the whole carry leaves
      o.frames = nullptr;
      o.F = 0;
      o.count = N;
      run = true;
    }
    if (run) {
      float* q = queue_reserve(c, (size_t)o.count);  // may move the queue (q_end changes)
      o.out = q + c->q_end;
      o.new_carry = static_cast<float*>(c->d_acc2.get(nb));
      o.new_nrm = use_norm ? static_cast<float*>(c->d_nrm2.get(nb)) : nullptr;
      check(launch_stream_ola(o, c->stream));
      if (!o.keep_carry) {
        check(cudaMemsetAsync(o.new_carry, 0, nb, c->stream));
        if (use_norm) check(cudaMemsetAsync(o.new_nrm, 0, nb, c->stream));
      }
      std::swap(c->d_acc.p, c->d_acc2.p);
      std::swap(c->d_acc.cap, c->d_acc2.cap);
      if (use_norm) {
        std::swap(c->d_nrm.p, c->d_nrm2.p);
        std::swap(c->d_nrm.cap, c->d_nrm2.cap);
      }
      c->q_end += (size_t)o.count;
    }
    return queue_emit(c, out_pcm, max_samples);
  } catch (...) {
    return 0;
  }
}

// ------------------------------------------------------------------ phase inference
struct PhaseCtx {
  uint32_t magic = 0x50484153u;
  int N = 0, hop = 0, half = 1, mode = 0, iterations = 0;
  void* fwd = nullptr;  // C2C forward context (mode 1)
  void* inv = nullptr;  // C2C inverse context (mode 1)
  DevBuf d_mag, d_spec, d_cep, d_re, d_im;  // mode 1 working set on the device
};

FFT_CFFI_API void* phase_init(int N, int hop, int half_spectrum, int mode, int iterations) {
  // fft_cffi.cpp:2065-2081
  if (N <= 0) return nullptr;
  PhaseCtx* p = new PhaseCtx();
  p->N = N;
  p->hop = hop > 0 ? hop : N;
  p->half = half_spectrum != 0;
  p->mode = mode;
  p->iterations = iterations;
  return p;
}

FFT_CFFI_API void phase_free(void* handle) {
  PhaseCtx* p = static_cast<PhaseCtx*>(handle);
  if (!p || p->magic != 0x50484153u) return;
  if (p->fwd) fft_free(p->fwd);
  if (p->inv) fft_free(p->inv);
  p->magic = 0;
  delete p;
}

FFT_CFFI_API size_t phase_infer_execute(void* handle, const float* in_mag, size_t frames,
                                        float* out_real, float* out_imag) {
  // fft_cffi.cpp:2083-2168
  PhaseCtx* p = static_cast<PhaseCtx*>(handle);
  if (!p || p->magic != 0x50484153u || !in_mag || !out_real || !out_imag || frames == 0) return 0;
  try {
    const int N = p->N;
    const int bins = p->half ? N / 2 + 1 : N;
    if (p->mode == 0) {
      // phase_infer.hpp:35-65: linear phase advance in FP64
      const double two_pi = 6.28318530717958647692;
      std::vector<double> dphi(bins), phi(bins, 0.0);
      for (int k = 0; k < bins; ++k) {
        const int kk = (k < N) ? k : (k % N);
        dphi[k] = two_pi * (double)kk * (double)p->hop / (double)N;
      }
      for (size_t f = 0; f < frames; ++f) {
        const size_t b = f * (size_t)bins;
        for (int k = 0; k < bins; ++k) {
          const double m = (double)in_mag[b + k];
          out_real[b + k] = (float)(m * std::cos(phi[k]));
          out_imag[b + k] = (float)(m * std::sin(phi[k]));
          phi[k] += dphi[k];
        }
      }
      return frames;
    }
    if (p->mode != 1) return 0;
    // Minimum phase from the real cepstrum, every step on the device: the
    // log-amplitude spectra, the inverse batch, the causal fold, the forward
    // batch and exp(L) per bin.
    if (!p->inv) p->inv = fft_init_full(N, 1, 1, 1, 0, 0, nullptr, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1);
    if (!p->fwd) p->fwd = fft_init_full(N, 1, 1, 0, 0, 0, nullptr, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1);
    if (!p->inv || !p->fwd) return 0;
    FftContext* ic = as_ctx(p->inv);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ic->device) cudaSetDevice(ic->device);
    struct Restore {
      int dev;
      ~Restore() {
        if (dev >= 0) cudaSetDevice(dev);
      }
    } restore{prev != ic->device ? prev : -1};
    auto ok = [](cudaError_t e) {
      if (e != cudaSuccess) throw std::runtime_error("cuda");
    };
    cudaStream_t st = ic->stream;
    const size_t nb = frames * (size_t)bins, nc = frames * (size_t)N;
    float* mag = static_cast<float*>(p->d_mag.get(nb * sizeof(float)));
    float2* spec = static_cast<float2*>(p->d_spec.get(nc * sizeof(float2)));
    float2* cep = static_cast<float2*>(p->d_cep.get(nc * sizeof(float2)));
    float* re = static_cast<float*>(p->d_re.get(nb * sizeof(float)));
    float* im = static_cast<float*>(p->d_im.get(nb * sizeof(float)));
    ok(cudaMemcpyAsync(mag, in_mag, nb * sizeof(float), cudaMemcpyDefault, st));
    ok(launch_minphase_log(mag, spec, (long long)frames, N, bins, p->half ? 1 : 0, st));
    ok(cudaStreamSynchronize(st));
    if (!fftfree_execute_c2c(p->inv, reinterpret_cast<const float*>(spec), reinterpret_cast<float*>(cep), frames))
      return 0;
    ok(cudaStreamSynchronize(ic->stream));
    ok(launch_minphase_fold(cep, (long long)frames, N, st));
    ok(cudaStreamSynchronize(st));
    if (!fftfree_execute_c2c(p->fwd, reinterpret_cast<const float*>(cep), reinterpret_cast<float*>(spec), frames))
      return 0;
    ok(cudaStreamSynchronize(as_ctx(p->fwd)->stream));
    ok(launch_minphase_exp(spec, re, im, (long long)frames, N, bins, st));
    ok(cudaMemcpyAsync(out_real, re, nb * sizeof(float), cudaMemcpyDefault, st));
    ok(cudaMemcpyAsync(out_imag, im, nb * sizeof(float), cudaMemcpyDefault, st));
    ok(cudaStreamSynchronize(st));
    return frames;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API int fft_griffin_lim(void* ctx_forward, void* ctx_inverse, const float* in_mag,
                                 size_t frames, int hop, int half_spectrum, int iterations,
                                 int pad_mode, unsigned int seed, float* out_real, float* out_imag) {
  // fft_cffi.cpp:2176-2248 and phase_infer.hpp:69-204
  if (!ctx_forward || !ctx_inverse || !in_mag || !out_real || !out_imag || frames == 0) return 0;
  if (in_mag == out_real || in_mag == out_imag || out_real == out_imag) return 0;
  FftContext* fc = as_ctx(ctx_forward);
  FftContext* ic = as_ctx(ctx_inverse);
  if (!fc || !ic) return 0;
  int cfgN = (ic->N > 0) ? ic->N : fc->N;
  if (cfgN <= 0) return 0;
  const bool half = half_spectrum != 0;
  if (half != (ic->half_spectrum != 0) || half != (fc->half_spectrum != 0)) return 0;
  int cfg_hop;
  if (hop > 0) cfg_hop = hop;
  else if (ic->hop > 0) cfg_hop = ic->hop;
  else if (fc->hop > 0) cfg_hop = fc->hop;
  else cfg_hop = cfgN;
  try {
    const size_t pf = fft_ctx_size(ctx_forward), pi = fft_ctx_size(ctx_inverse);
    size_t plan_n = pf ? pf : pi;
    if (plan_n == 0) plan_n = (size_t)cfgN;
    if (pi && pf && pi != pf) plan_n = pi;
    const size_t bins = half ? plan_n / 2 + 1 : plan_n;
    const size_t total_bins = bins * frames;
    const size_t hp = (size_t)cfg_hop;
    const size_t ola_len = (frames - 1) * hp + plan_n;
    const int iters = (iterations > 0) ? iterations : 32;
    // Initial phases as the reference draws them (phase_infer.hpp:128-138):
    // std::mt19937 and a float uniform in [-pi, pi), in order on the host.
    // Their cosines and sines (std::cos / std::sin of the float angle, as
    // there) are evaluated by several host threads; the device multiplies
    // them by the magnitudes.
    // Both contexts are this call's for its duration (the forward one holds
    // the working set), taken together so that no two calls deadlock.
    std::scoped_lock lk(fc->mu, ic->mu);
    if (fc->h_gl_cs_cap < total_bins) {
      if (fc->h_gl_cs) cudaFreeHost(fc->h_gl_cs);
      fc->h_gl_cs = nullptr;
      fc->h_gl_cs_cap = 0;
      void* hp_cs = nullptr;
      if (cudaHostAlloc(&hp_cs, total_bins * sizeof(float2), cudaHostAllocPortable) != cudaSuccess) return 0;
      fc->h_gl_cs = static_cast<float2*>(hp_cs);
      fc->h_gl_cs_cap = total_bins;
    }
    float2* cs = fc->h_gl_cs;
    using clk = std::chrono::steady_clock;
    const clk::time_point t_start = clk::now();
    // The iterations run on the device (phase_infer.hpp:140-208): the inverse
    // batch, the count-normalised overlap-add, and the forward STFT whose
    // epilogue projects its spectra onto the target magnitudes, all enqueued
    // without host synchronisation; the two contexts' streams are ordered by
    // events when they differ.
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != fc->device) cudaSetDevice(fc->device);
    struct Restore {
      int dev;
      ~Restore() {
        if (dev >= 0) cudaSetDevice(dev);
      }
    } restore{prev != fc->device ? prev : -1};
    const size_t fb = total_bins * sizeof(float);
    float* mag = static_cast<float*>(fc->d_gl_spec.get(3 * fb));
    float* re = mag + total_bins;
    float* im = re + total_bins;
    // forward outputs of the unfused projection; first the cosines and sines
    float* tr = static_cast<float*>(fc->d_gl_tmp.get(3 * fb));
    float* ti = tr + total_bins;
    float* tm = ti + total_bins;
    float* frame_pcm = static_cast<float*>(fc->d_gl_frames.get(frames * plan_n * sizeof(float)));
    float* ola = static_cast<float*>(fc->d_gl_ola.get(ola_len * sizeof(float)));
    cudaStream_t st = fc->stream;
    cudaStream_t ist = ic->stream;
    auto ok = [](cudaError_t e) {
      if (e != cudaSuccess) throw std::runtime_error("cuda");
    };
    struct Events {
      cudaEvent_t inv = nullptr, fwd = nullptr;
      ~Events() {
        if (inv) cudaEventDestroy(inv);
        if (fwd) cudaEventDestroy(fwd);
      }
    } ev;
    const bool two = ist != st;
    if (two) {
      ok(cudaEventCreateWithFlags(&ev.inv, cudaEventDisableTiming));
      ok(cudaEventCreateWithFlags(&ev.fwd, cudaEventDisableTiming));
    }
    ok(cudaMemcpyAsync(mag, in_mag, fb, cudaMemcpyDefault, st));
    if (!gl_initial_phasors(seed ? seed : 0x47d7bfad, total_bins, fc->h_gl_state, cs,
                            reinterpret_cast<float2*>(tr), fc->device, st))
      throw std::runtime_error("cuda");
    const clk::time_point t_phasors = clk::now();
    ok(launch_gl_init(mag, reinterpret_cast<const float2*>(tr), re, im, (long long)total_bins, st));
    ok(cudaStreamSynchronize(st));
    const clk::time_point t_upload = clk::now();
    // The reference refines out_real/out_imag in place, so a failed pass
    // leaves the spectra of the last completed one there.
    auto flush = [&]() {
      if (two) ok(cudaStreamSynchronize(ist));
      ok(cudaMemcpyAsync(out_real, re, fb, cudaMemcpyDefault, st));
      ok(cudaMemcpyAsync(out_imag, im, fb, cudaMemcpyDefault, st));
      ok(cudaStreamSynchronize(st));
    };
    OlaArgs o{};
    o.frames_buf = frame_pcm;
    o.frames = (long long)frames;
    o.N = (int)plan_n;
    o.H = (int)hp;
    o.cola = 1;  // divide by the number of frames covering the sample
    o.weight = nullptr;
    o.out = ola;
    o.len = (long long)ola_len;  // every sample written: no clearing
    for (int it = 0; it < iters; ++it) {
      size_t pr = 0, ff = 0;
      try {
        if (two && it > 0) ok(cudaStreamWaitEvent(ist, ev.fwd, 0));
        pr = gl_inverse_enqueue(ic, re, im, frames, frame_pcm);
        if (pr != 0) {
          if (two) {
            ok(cudaEventRecord(ev.inv, ist));
            ok(cudaStreamWaitEvent(st, ev.inv, 0));
          }
          o.frames = (long long)std::min(pr, frames);
          ok(launch_ola(o, st, &fc->launches));
          ff = gl_forward_project_enqueue(fc, ola, ola_len, pad_mode, frames, mag, re, im, (int)bins, half,
                                          (plan_n & 1) == 0, tr, ti, tm);
          if (two) ok(cudaEventRecord(ev.fwd, st));
        }
      } catch (...) {
        pr = 0;
      }
      if (pr == 0 || ff == 0) {
        flush();
        return 0;
      }
    }
    const clk::time_point t_enqueued = clk::now();
    flush();
    if (verbose()) {
      auto ms = [](clk::time_point a, clk::time_point b) {
        return std::chrono::duration<double, std::milli>(b - a).count();
      };
      std::fprintf(stderr,
                   "[diag] fft_griffin_lim: %zu bins x %d iterations: phasors %.3f ms, upload %.3f ms, "
                   "enqueue %.3f ms, drain + copy-out %.3f ms\n",
                   total_bins, iters, ms(t_start, t_phasors), ms(t_phasors, t_upload), ms(t_upload, t_enqueued),
                   ms(t_enqueued, clk::now()));
    }
    return 1;
  } catch (...) {
    return 0;
  }
}

}  // extern "C"
