// abi.cpp -- the reference C ABI (fft_cffi.hpp) implemented over CUDA.
//
// Host logic (validation, frame counting, window construction, streaming
// buffers, Griffin-Lim / phase inference drivers, the recovery coordinator)
// follows the reference's fft_cffi.cpp line by line where behaviour is
// observable through the ABI; every transform runs on the GPU through
// kernels.cu.  There is no CPU fallback: without a usable CUDA device the
// init functions print an error and return NULL.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/fft_cffi.h"
#include "../../include/fftfree_b200.h"
#include "context.h"
#include "kernels.h"
#include "recovery.h"

namespace ffb {

int run_meta(FftContext* c, const float* in, float* out, size_t batch, const fftfree_metadata_request* reqs,
             int nreq);

// ------------------------------------------------------------------ utilities
static bool verbose() {
  static const bool v = [] {
    const char* e = std::getenv("FFTFREE_VERBOSE");
    return e && *e && e[0] != '0';
  }();
  return v;
}

#define FFB_CHECK(expr)                                                              \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess) {                                                         \
      std::fprintf(stderr, "[fftfree_b200] CUDA error %s at %s:%d: %s\n",            \
                   cudaGetErrorName(_e), __FILE__, __LINE__, cudaGetErrorString(_e)); \
      throw std::runtime_error("cuda");                                              \
    }                                                                                \
  } while (0)

void* DevBuf::get(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (bytes > cap) {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      p = nullptr;
      throw std::runtime_error("cudaMalloc failed");
    }
    cap = bytes;
  }
  return p;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

FftContext* as_ctx(void* h) {
  FftContext* c = static_cast<FftContext*>(h);
  if (!c || c->magic != 0x46465442u) return nullptr;
  return c;
}

PostFlags FftContext::post_flags() const {
  PostFlags pf{};
  const int m = eff_transform();
  pf.r2c_half = (m == 1 && half_spectrum) ? 1 : 0;
  pf.polar = store_polar ? 1 : 0;
  pf.reduce = (!store_polar && reduce_magnitude) ? 1 : 0;
  pf.clear_imag = (m == 2 && !store_polar && !reduce_magnitude) ? 1 : 0;
  return pf;
}

static bool is_pow2(size_t v) { return v != 0 && (v & (v - 1)) == 0; }
static size_t next_pow2(size_t v) {
  if (v <= 1) return 1;
  size_t p = 1;
  while (p < v) p <<= 1;
  return p;
}
static int ilog2(size_t v) {
  int l = 0;
  while (((size_t)1 << l) < v) ++l;
  return l;
}

static bool device_available_impl() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return false;
  }
  return true;
}

static bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Input: device pointers are used in place; host data is copied into `buf`.
static const float* stage_in(FftContext* c, DevBuf& buf, const float* src, size_t count) {
  if (is_device_ptr(src)) return src;
  float* d = static_cast<float*>(buf.get(count * sizeof(float)));
  if (count) FFB_CHECK(cudaMemcpyAsync(d, src, count * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  return d;
}

struct OutTarget {
  float* user = nullptr;
  float* dev = nullptr;
  size_t count = 0;
  bool host = false;
};

static OutTarget stage_out(DevBuf& buf, float* user, size_t count) {
  OutTarget o;
  o.user = user;
  o.count = count;
  if (is_device_ptr(user)) {
    o.dev = user;
  } else {
    o.host = true;
    o.dev = static_cast<float*>(buf.get(count * sizeof(float)));
  }
  return o;
}

static void finish_out(FftContext* c, const OutTarget& o) {
  if (o.host && o.count)
    FFB_CHECK(cudaMemcpyAsync(o.user, o.dev, o.count * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
}

static void finish_call(FftContext* c, bool any_host) {
  FFB_CHECK(cudaGetLastError());
  if (any_host || !c->async) FFB_CHECK(cudaStreamSynchronize(c->stream));
}

// ------------------------------------------------------------------ windows
// fft_cffi.cpp:163-208
static void normalize_window(std::vector<float>& w, int policy) {
  if (w.empty()) return;
  if (policy == FFT_WINDOW_NORM_L2) {
    double s2 = 0.0;
    for (float v : w) s2 += double(v) * double(v);
    s2 = std::sqrt(std::max(1e-30, s2));
    if (s2 > 0) for (auto& v : w) v = float(v / s2);
  } else if (policy == FFT_WINDOW_NORM_AREA) {
    double s = 0.0;
    for (float v : w) s += double(v);
    if (std::abs(s) > 1e-30) for (auto& v : w) v = float(v / s);
  }
}

static std::vector<float> build_window(int kind, int W, float p1, float /*p2*/) {
  std::vector<float> w(W > 0 ? W : 0, 1.0f);
  if (W <= 0) return w;
  const double pi = 3.141592653589793238462643383279502884;
  switch (kind) {
    case FFT_WINDOW_HANN:
    case FFT_WINDOW_KAISER:  // Hann placeholder in the reference (fft_cffi.cpp:200-203)
      for (int n = 0; n < W; ++n) w[n] = float(0.5 * (1.0 - std::cos(2.0 * pi * n / (W - 1))));
      break;
    case FFT_WINDOW_HAMMING:
      for (int n = 0; n < W; ++n) w[n] = float(0.54 - 0.46 * std::cos(2.0 * pi * n / (W - 1)));
      break;
    case FFT_WINDOW_BLACKMAN:
      for (int n = 0; n < W; ++n)
        w[n] = float(0.42 - 0.5 * std::cos(2.0 * pi * n / (W - 1)) + 0.08 * std::cos(4.0 * pi * n / (W - 1)));
      break;
    case FFT_WINDOW_TUKEY: {
      const double alpha = (p1 == 0.0f ? 0.5 : p1);
      const int L = std::max(1, W - 1);
      for (int n = 0; n < W; ++n) {
        const double x = double(n) / double(L);
        if (x < alpha / 2) w[n] = float(0.5 * (1 + std::cos(pi * (2 * x / alpha - 1))));
        else if (x <= 1 - alpha / 2) w[n] = 1.0f;
        else w[n] = float(0.5 * (1 + std::cos(pi * (2 * x / alpha - 2 / alpha + 1))));
      }
      break;
    }
    default:
      break;
  }
  return w;
}

std::vector<float> window_taps(int kind, int W, float p1, float p2, int norm_policy) {
  std::vector<float> w = build_window(kind, W, p1, p2);
  normalize_window(w, norm_policy);
  return w;
}

static void upload_windows(FftContext* c) {
  if (!c->windows_enabled || c->windows_uploaded) return;
  const size_t n = (size_t)c->N;
  std::vector<float> wa(n, 1.0f), ws(n, 1.0f), wgt(n, 1.0f);
  for (size_t i = 0; i < n; ++i) {
    wa[i] = i < c->analysis_win.size() ? c->analysis_win[i] : 1.0f;
    ws[i] = i < c->synthesis_win.size() ? c->synthesis_win[i] : 1.0f;
    wgt[i] = wa[i] * ws[i];  // cola_window_weight (fft_cffi.cpp:210-226)
  }
  float* da = static_cast<float*>(c->d_analysis.get(n * 4));
  float* ds = static_cast<float*>(c->d_synthesis.get(n * 4));
  float* dw = static_cast<float*>(c->d_weight.get(n * 4));
  FFB_CHECK(cudaMemcpyAsync(da, wa.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  FFB_CHECK(cudaMemcpyAsync(ds, ws.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  FFB_CHECK(cudaMemcpyAsync(dw, wgt.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
  FFB_CHECK(cudaStreamSynchronize(c->stream));
  c->windows_uploaded = true;
}

// ------------------------------------------------------------------ plans
static int requested_logr(const FftContext* c) {
  auto lg = [](int r) { return r == 4 ? 2 : r == 8 ? 3 : r == 16 ? 4 : -1; };
  int best = -1;
  for (int r : c->radix_pattern) best = std::max(best, lg(r));
  if (best >= 0) return best;
  return lg(c->radix);
}

// Transform sizes the kernels cover (single pass up to 2^13 complex points,
// multi-pass beyond, up to 2^20).
static bool size_supported(int N, bool real_input) {
  (void)real_input;
  return ilog2((size_t)N) <= max_multi_pass_log();
}

static bool single_pass(int N, bool real_input) {
  const int lg = ilog2((size_t)N);
  const int logm = real_input ? std::max(0, lg - 1) : lg;
  return logm <= max_single_pass_log();
}

static float2* scratch_for(FftContext* c, int N, long long batch, size_t* chunk) {
  *chunk = four_step_chunk(ilog2((size_t)N), batch);
  // two slots when the multi-pass pipeline alternates between chunks,
  // one when a single chunk covers the batch
  const size_t slots = ((long long)*chunk < batch) ? 2 : 1;
  return static_cast<float2*>(c->d_scratch.get(slots * *chunk * (size_t)N * sizeof(float2)));
}

static void setup_device(FftContext* c) {
  FFB_CHECK(cudaGetDevice(&c->device));
  FFB_CHECK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
  c->stream = c->own_stream;
  (void)twiddle_pyramid(ilog2((size_t)std::max(c->N, 1)) + 1, c->stream);
  if (!twiddle_pass_tables(c->stream)) throw std::runtime_error("twiddle tables");
  upload_windows(c);
}

static size_t frame_count(const FftContext* c, size_t pcm_len, int pad_mode, size_t max_frames) {
  // fft_cffi.cpp:710-750
  const int N = c->N;
  if (N <= 0) return 0;
  const int W = c->window ? c->window : N;
  const int H = c->hop ? c->hop : W;
  if (W <= 0 || H <= 0) return 0;
  if (W > N) return 0;
  const int eff = (pad_mode == 0) ? c->pad_mode : pad_mode;
  size_t frames = 0;
  if (pcm_len < (size_t)W) {
    if (eff == 1) frames = 1;
    else return 0;
  } else {
    frames = 1 + (pcm_len - (size_t)W) / (size_t)H;
    const size_t last = (frames - 1) * (size_t)H;
    const size_t remaining = (pcm_len > last) ? pcm_len - last : 0;
    if (remaining < (size_t)W) {
      if (eff == 1) {
      } else if (eff == 2) {
        if (frames > 0) frames -= 1;
      } else {
        return 0;
      }
    }
  }
  if (frames == 0) return 0;
  if (max_frames != 0 && frames > max_frames) frames = max_frames;
  return frames;
}

// ------------------------------------------------------------------ host pipeline
// A call on host buffers is cut into chunks whose upload (up_stream),
// kernels (the context stream) and download (down_stream) overlap: chunk
// i + 1 uploads while chunk i computes and chunk i - 1 downloads, both
// directions of the host link busy at once.  Pinned host memory lets the
// copies run asynchronously; pageable memory still works, with less overlap.
constexpr size_t kPipeChunkBytes = 32u << 20;  // host bytes moved per chunk, about
constexpr int kPipeMaxChunks = 16;

static int pipe_chunks(size_t host_bytes, long long units) {
  if (host_bytes < 2 * kPipeChunkBytes || units < 2) return 1;
  long long n = (long long)(host_bytes / kPipeChunkBytes);
  n = std::min<long long>(std::min<long long>(n, kPipeMaxChunks), units);
  return (int)std::max<long long>(n, 1);
}

static void ensure_pipe(FftContext* c) {
  if (c->up_stream) return;
  FFB_CHECK(cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking));
  FFB_CHECK(cudaStreamCreateWithFlags(&c->down_stream, cudaStreamNonBlocking));
  c->pipe_events.assign(2 * kPipeMaxChunks + 2, nullptr);
  for (cudaEvent_t& e : c->pipe_events) FFB_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

// Runs `chunks` pieces: up(i, s) enqueues piece i's host->device copies,
// run(i, s) its kernels, down(i, s) its device->host copies.  On return the
// context stream is ordered after every copy; the caller synchronises it.
template <class Up, class Run, class Down>
static void run_pipelined(FftContext* c, int chunks, Up&& up, Run&& run, Down&& down) {
  ensure_pipe(c);
  cudaEvent_t* ev = c->pipe_events.data();
  cudaEvent_t start = ev[2 * kPipeMaxChunks], done = ev[2 * kPipeMaxChunks + 1];
  FFB_CHECK(cudaEventRecord(start, c->stream));
  FFB_CHECK(cudaStreamWaitEvent(c->up_stream, start, 0));
  FFB_CHECK(cudaStreamWaitEvent(c->down_stream, start, 0));
  for (int i = 0; i < chunks; ++i) {
    up(i, c->up_stream);
    FFB_CHECK(cudaEventRecord(ev[2 * i], c->up_stream));
    FFB_CHECK(cudaStreamWaitEvent(c->stream, ev[2 * i], 0));
    run(i, c->stream);
    FFB_CHECK(cudaEventRecord(ev[2 * i + 1], c->stream));
    FFB_CHECK(cudaStreamWaitEvent(c->down_stream, ev[2 * i + 1], 0));
    down(i, c->down_stream);
  }
  FFB_CHECK(cudaEventRecord(done, c->down_stream));
  FFB_CHECK(cudaStreamWaitEvent(c->stream, done, 0));
}

static void copy_h2d(float* dst, const float* src, size_t count, cudaStream_t s) {
  if (count) FFB_CHECK(cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyHostToDevice, s));
}
static void copy_d2h(float* dst, const float* src, size_t count, cudaStream_t s) {
  if (count) FFB_CHECK(cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyDeviceToHost, s));
}

// STFT of `frames` frames of `pcm` into (re, im, mag), bins per frame
// `out_bins`; shared by fft_execute_batched, fft_execute and the one-shot.
static void run_stft(FftContext* c, const float* pcm, size_t pcm_len, size_t frames, int W, int H,
                     bool use_window, int out_bins, bool mag_from_real, const PostFlags& pf,
                     bool mirror, float* re, float* im, float* mag) {
  const size_t span = std::min(pcm_len, (frames - 1) * (size_t)H + (size_t)W);
  const bool in_host = !is_device_ptr(pcm);
  const size_t outn = frames * (size_t)out_bins;
  OutTarget o_re = stage_out(c->d_out0, re, outn);
  OutTarget o_im = stage_out(c->d_out1, im, outn);
  OutTarget o_mag = stage_out(c->d_out2, mag, outn);
  const bool any_host = in_host || o_re.host || o_im.host || o_mag.host;
  const size_t host_bytes = ((in_host ? span : 0) +
                             outn * ((o_re.host ? 1 : 0) + (o_im.host ? 1 : 0) + (o_mag.host ? 1 : 0))) * 4;
  const int chunks = single_pass(c->N, true) ? pipe_chunks(host_bytes, (long long)frames) : 1;
  // host input is uploaded here, or chunk by chunk by the pipeline below
  const float* d_pcm = (chunks > 1 && in_host) ? static_cast<const float*>(c->d_in0.get(span * sizeof(float)))
                                               : stage_in(c, c->d_in0, pcm, span);
  StftArgs a{};
  a.pcm = d_pcm;
  a.pcm_len = (long long)span;
  a.frames = (long long)frames;
  a.N = c->N;
  a.W = W;
  a.H = H;
  a.win = (use_window && c->windows_enabled) ? static_cast<const float*>(c->d_analysis.p) : nullptr;
  a.mirror = mirror ? 1 : 0;
  a.inverse = c->inverse ? 1 : 0;
  a.pf = pf;
  a.out_bins = out_bins;
  a.out_stride = out_bins;
  a.mag_from_real = mag_from_real ? 1 : 0;
  a.out_re = o_re.dev;
  a.out_im = o_im.dev;
  a.out_mag = o_mag.dev;
  if (chunks > 1) {
    // frames [f0, f1) of chunk i read pcm[f0*H, (f1-1)*H + W); uploads skip
    // what an earlier chunk already brought over
    const size_t per = (frames + chunks - 1) / chunks;
    float* d_in = const_cast<float*>(d_pcm);
    size_t uploaded = 0;
    auto range = [&](int i, size_t* f0, size_t* f1) {
      *f0 = std::min(frames, (size_t)i * per);
      *f1 = std::min(frames, *f0 + per);
    };
    run_pipelined(
        c, chunks,
        [&](int i, cudaStream_t s) {
          size_t f0, f1;
          range(i, &f0, &f1);
          if (!in_host || f1 <= f0) return;
          const size_t hi = std::min(span, (f1 - 1) * (size_t)H + (size_t)W);
          const size_t lo = std::max(uploaded, f0 * (size_t)H);
          if (hi > lo) copy_h2d(d_in + lo, pcm + lo, hi - lo, s);
          uploaded = std::max(uploaded, hi);
        },
        [&](int i, cudaStream_t s) {
          size_t f0, f1;
          range(i, &f0, &f1);
          if (f1 <= f0) return;
          StftArgs b = a;
          b.pcm = d_pcm + f0 * (size_t)H;
          b.pcm_len = (long long)(span - f0 * (size_t)H);
          b.frames = (long long)(f1 - f0);
          b.out_re = a.out_re + f0 * (size_t)out_bins;
          b.out_im = a.out_im + f0 * (size_t)out_bins;
          b.out_mag = a.out_mag + f0 * (size_t)out_bins;
          FFB_CHECK(launch_stft(b, c->logr_req, s, &c->launches));
        },
        [&](int i, cudaStream_t s) {
          size_t f0, f1;
          range(i, &f0, &f1);
          const size_t o = f0 * (size_t)out_bins, n = (f1 - f0) * (size_t)out_bins;
          for (const OutTarget* t : {&o_re, &o_im, &o_mag})
            if (t->host) copy_d2h(t->user + o, t->dev + o, n, s);
        });
    finish_call(c, true);
    return;
  }
  if (single_pass(c->N, true)) {
    FFB_CHECK(launch_stft(a, c->logr_req, c->stream, &c->launches));
  } else {
    size_t chunk = 0;
    float2* scratch = scratch_for(c, c->N, (long long)frames, &chunk);
    FFB_CHECK(launch_four_step_stft(a, scratch, chunk, c->stream, &c->launches));
  }
  finish_out(c, o_re);
  finish_out(c, o_im);
  finish_out(c, o_mag);
  finish_call(c, any_host);
}

static bool stft_mirror(const FftContext* c) {
  return !c->stockham() && c->eff_transform() == 2 && c->half_spectrum;
}

// Complex/inverse batch into `out` (frames x N) or, with OLA, into `out`
// as frames*N samples.
static void run_complex_batch(FftContext* c, const float* in_re, const float* in_im, size_t frames,
                              float* out_pcm, const std::vector<char>* raw_frames) {
  const int N = c->N;
  const int bins = c->bins();
  const size_t inn = frames * (size_t)bins;
  bool any_host = !is_device_ptr(in_re) || !is_device_ptr(in_im);
  const float* d_re = stage_in(c, c->d_in0, in_re, inn);
  const float* d_im = stage_in(c, c->d_in1, in_im, inn);
  const size_t outn = frames * (size_t)N;
  OutTarget o = stage_out(c->d_out0, out_pcm, outn);
  any_host = any_host || o.host;
  CplxBatchArgs a{};
  a.in_re = d_re;
  a.in_im = d_im;
  a.frames = (long long)frames;
  a.N = N;
  a.bins = bins;
  const int m = c->eff_transform();
  a.c2r_half = (c->half_spectrum && m == 2) ? 1 : 0;
  a.ct_pre = c->stockham() ? 0 : (m == 1 ? 1 : ((m == 2 && c->half_spectrum) ? 2 : 0));
  a.polar_in = c->store_polar ? 1 : 0;
  a.inverse = c->inverse ? 1 : 0;
  a.pf = c->post_flags();
  a.synth = c->windows_enabled ? static_cast<const float*>(c->d_synthesis.p) : nullptr;
  float* frames_out = c->apply_ola ? static_cast<float*>(c->d_frames.get(outn * sizeof(float))) : o.dev;
  a.out = frames_out;
  if (single_pass(N, a.c2r_half && N >= 4)) {
    FFB_CHECK(launch_cplx_batch(a, c->logr_req, c->stream, &c->launches));
  } else {
    size_t chunk = 0;
    float2* scratch = scratch_for(c, N, (long long)frames, &chunk);
    FFB_CHECK(launch_four_step_cplx(a, scratch, chunk, c->stream, &c->launches));
  }
  if (raw_frames) {
    // Frames the recovery coordinator gave up on keep the restored
    // (untransformed) column: its real part times the synthesis window.
    std::vector<float> hre(inn), him(inn), row(N);
    FFB_CHECK(cudaMemcpyAsync(hre.data(), d_re, inn * 4, cudaMemcpyDeviceToHost, c->stream));
    FFB_CHECK(cudaStreamSynchronize(c->stream));
    std::vector<float> synth(c->synthesis_win);
    for (size_t f = 0; f < frames; ++f) {
      if (!(*raw_frames)[f]) continue;
      for (int i = 0; i < N; ++i) {
        float v = 0.f;
        if (i < bins) v = hre[f * bins + i];
        else if (a.c2r_half) v = hre[f * bins + (N - i)];
        if (c->windows_enabled && (size_t)i < synth.size()) v *= synth[i];
        row[i] = v;
      }
      FFB_CHECK(cudaMemcpyAsync(frames_out + f * N, row.data(), N * 4, cudaMemcpyHostToDevice, c->stream));
      FFB_CHECK(cudaStreamSynchronize(c->stream));
    }
  }
  if (c->apply_ola) {
    OlaArgs ola{};
    ola.frames_buf = frames_out;
    ola.frames = (long long)frames;
    ola.N = N;
    ola.H = (c->hop > 0) ? c->hop : ((c->window > 0) ? c->window : N);
    ola.cola = (c->cola_mode == FFT_COLA_NORMALIZE) ? 1 : 0;
    ola.weight = c->windows_enabled ? static_cast<const float*>(c->d_weight.p) : nullptr;
    ola.out = o.dev;
    FFB_CHECK(launch_ola(ola, c->stream, &c->launches));
  }
  finish_out(c, o);
  finish_call(c, any_host);
}

// ------------------------------------------------------------------ Griffin-Lim steps
// The two transforms of one Griffin-Lim iteration (phase_infer.hpp:140-197)
// on device buffers, enqueued on the context's stream without host
// synchronisation; the loop orders the two contexts' streams itself.
namespace {
struct AsyncScope {
  FftContext* c;
  bool was;
  explicit AsyncScope(FftContext* ctx) : c(ctx), was(ctx->async) { c->async = true; }
  ~AsyncScope() { c->async = was; }
};
}  // namespace

size_t gl_inverse_enqueue(FftContext* c, const float* re, const float* im, size_t frames, float* frame_pcm) {
  // fft_execute_complex_batched without recovery (fft_cffi.cpp:1042-1340)
  if (c->N <= 0 || frames == 0) return 0;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  DeviceGuard g(c->device);
  AsyncScope as(c);
  run_complex_batch(c, re, im, frames, frame_pcm, nullptr);
  return frames;
}

size_t gl_forward_project_enqueue(FftContext* c, const float* pcm, size_t pcm_len, int pad_mode,
                                  size_t max_frames, const float* mag, float* re, float* im, int bins,
                                  bool half, bool even_n, float* tr, float* ti, float* tm) {
  // fft_execute_batched without recovery (fft_cffi.cpp:701-1034), then
  // re + i im = mag e^{i arg} over the frames it produced
  // (phase_infer.hpp:182-207)
  const size_t frames = frame_count(c, pcm_len, pad_mode, max_frames);
  if (frames == 0) return 0;
  const int W = c->window ? c->window : c->N;
  const int H = c->hop ? c->hop : W;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  DeviceGuard g(c->device);
  const PostFlags pf = c->post_flags();
  const size_t upd = std::min(frames, max_frames ? max_frames : frames);
  if (c->bins() == bins && !pf.polar && !pf.reduce && single_pass(c->N, true) && is_device_ptr(pcm)) {
    // one launch: the STFT's epilogue writes the projected spectra
    StftArgs a{};
    a.pcm = pcm;
    a.pcm_len = (long long)std::min(pcm_len, (frames - 1) * (size_t)H + (size_t)W);
    a.frames = (long long)upd;
    a.N = c->N;
    a.W = W;
    a.H = H;
    a.win = c->windows_enabled ? static_cast<const float*>(c->d_analysis.p) : nullptr;
    a.mirror = stft_mirror(c) ? 1 : 0;
    a.inverse = c->inverse ? 1 : 0;
    a.pf = pf;
    a.out_bins = bins;
    a.out_stride = bins;
    a.out_re = re;
    a.out_im = im;
    a.out_mag = tm;
    a.mag_only = 4;
    a.target = mag;
    FFB_CHECK(launch_stft(a, c->logr_req, c->stream, &c->launches));
    FFB_CHECK(cudaGetLastError());
    return frames;
  }
  {
    AsyncScope as(c);
    run_stft(c, pcm, pcm_len, frames, W, H, true, c->bins(), true, pf, stft_mirror(c), tr, ti, tm);
  }
  FFB_CHECK(launch_gl_project(mag, tr, ti, re, im, (long long)(upd * (size_t)bins), bins, half ? 1 : 0,
                              even_n ? 1 : 0, c->stream));
  return frames;
}

}  // namespace ffb

using namespace ffb;

// ====================================================================== ABI
extern "C" {

FFT_CFFI_API int fftfree_device_available(void) { return device_available_impl() ? 1 : 0; }

static FftContext* new_context_or_null() {
  if (!device_available_impl()) {
    std::fprintf(stderr,
                 "[fftfree_b200] no usable CUDA device: this library runs every transform on the "
                 "GPU and has no CPU fallback\n");
    return nullptr;
  }
  return new FftContext();
}

static int env_default_kernel_override() {
  // fft_cffi.cpp:104-159 (token parsing and the value it yields)
  static const int cached = [] {
    const char* env = std::getenv("FFTFREE_DEFAULT_KERNEL");
    if (!env) return 0;
    std::string s(env);
    auto b = s.find_first_not_of(" \t\r\n");
    auto e = s.find_last_not_of(" \t\r\n");
    s = (b == std::string::npos) ? std::string() : s.substr(b, e - b + 1);
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    if (s.empty() || s == "0" || s == "auto" || s == "default") return 0;
    if (s == "cooleytukey" || s == "cooley" || s == "cooley-tukey" || s == "cooley_tukey" || s == "ct")
      return (int)FFT_KERNEL_COOLEYTUKEY;
    if (s == "stockham" || s == "stock" || s == "sh") return (int)FFT_KERNEL_STOCKHAM;
    if (s == "external" || s == "ext" || s == "custom") return (int)FFT_KERNEL_EXTERNAL;
    char* end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    if (end && *end == '\0' && (v == 0 || v == 1 || v == 2)) return (int)v;
    return 0;
  }();
  return cached;
}

FFT_CFFI_API void* fft_init_ex(size_t n, int threads, int lanes, int inverse, int kernel, int radix,
                               const int* radix_pattern, size_t radix_pattern_len, int pad_mode,
                               int window, int hop) {
  // fft_cffi.cpp:540-658
  try {
    if (n == 0) return nullptr;
    size_t plan_n = n;
    if (!is_pow2(plan_n)) {
      if (pad_mode == 1) {
        plan_n = next_pow2(plan_n);
      } else {
        std::fprintf(stderr,
                     "fft_init: refusing to auto-pad N=%zu -> %zu because pad_mode!=ALWAYS; set "
                     "pad_mode=1 to permit padding or supply power-of-two N\n",
                     n, next_pow2(n));
        return nullptr;
      }
    }
    if (plan_n > (size_t)INT_MAX || !size_supported((int)plan_n, true)) {
      std::fprintf(stderr, "[fftfree_b200] fft_init: N=%zu exceeds the supported transform size\n", plan_n);
      return nullptr;
    }
    FftContext* c = new_context_or_null();
    if (!c) return nullptr;
    c->N = (int)plan_n;
    c->inverse = inverse != 0;
    c->kernel = kernel;
    if (c->kernel == 0) {
      const int ek = env_default_kernel_override();
      if (ek != 0) c->kernel = ek;
    }
    c->radix = radix;
    c->pad_mode = pad_mode;
    c->window = window;
    c->hop = hop;
    if (radix_pattern && radix_pattern_len > 0)
      c->radix_pattern.assign(radix_pattern, radix_pattern + radix_pattern_len);
    c->threads = threads > 0 ? threads : 4;  // Plan::Limits::kDefaultRuntimeThreads
    c->lanes = lanes > 0 ? lanes : 0;
    c->has_pool = false;  // fft_init_ex creates no WorkerPool
    c->logr_req = requested_logr(c);
    try {
      setup_device(c);
    } catch (...) {
      delete c;
      return nullptr;
    }
    return c;
  } catch (...) {
    std::fprintf(stderr, "fft_init: unknown exception caught, returning NULL\n");
    return nullptr;
  }
}

FFT_CFFI_API void* fft_init(size_t n, int threads, int lanes, int inverse, int kernel, int radix,
                            const int* radix_pattern, size_t radix_pattern_len, int pad_mode) {
  return fft_init_ex(n, threads, lanes, inverse, kernel, radix, radix_pattern, radix_pattern_len,
                     pad_mode, 0, 0);
}

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
                                    int window_norm_policy, int cola_mode) {
  // fft_cffi.cpp:1824-1978.  The reference installs POSIX crash handlers
  // here; a CUDA process keeps its own signal handling, so this build does
  // not (save_crash_logs / silent_crash_reports are accepted and ignored).
  (void)save_crash_logs;
  (void)silent_crash_reports;
  try {
    // The Plan constructor rejects non-power-of-two N (eigen_fft.hpp:2229-2232);
    // N == 0 never returns there, here it is rejected.
    if (n == 0 || !is_pow2(n) || n > (size_t)INT_MAX) {
      if (verbose()) std::fprintf(stderr, "[error] fft_init_full: N must be a power of two\n");
      return nullptr;
    }
    if (!size_supported((int)n, true)) {
      std::fprintf(stderr, "[fftfree_b200] fft_init_full: N=%zu exceeds the supported transform size\n", n);
      return nullptr;
    }
    FftContext* c = new_context_or_null();
    if (!c) return nullptr;
    c->N = (int)n;
    c->inverse = inverse != 0;
    c->kernel = kernel;
    c->radix = radix;
    c->pad_mode = pad_mode;
    c->window = window;
    c->hop = hop;
    c->transform = transform;
    c->reduce_magnitude = reduce_magnitude;
    c->store_polar = store_polar;
    c->half_spectrum = half_spectrum;
    c->allow_outer_parallel = allow_outer_parallel;
    c->allow_inner_parallel = allow_inner_parallel;
    c->inner_threads = inner_threads;
    c->analysis_win_kind = analysis_window_kind;
    c->synthesis_win_kind = synthesis_window_kind;
    c->win_param1 = analysis_param1;
    c->win_param2 = analysis_param2;
    c->win_norm_policy = window_norm_policy;
    c->cola_mode = cola_mode;
    c->windows_enabled = apply_windows != 0;
    const int useW = (window > 0) ? window : c->N;
    {
      auto aw = build_window(analysis_window_kind, useW, analysis_param1, analysis_param2);
      normalize_window(aw, window_norm_policy);
      c->analysis_win.assign(c->N, 1.0f);
      for (int i = 0; i < useW && i < c->N; ++i) c->analysis_win[i] = aw[i];
    }
    {
      auto sw = build_window(synthesis_window_kind, useW, synthesis_param1, synthesis_param2);
      normalize_window(sw, window_norm_policy);
      c->synthesis_win.assign(c->N, 1.0f);
      for (int i = 0; i < useW && i < c->N; ++i) c->synthesis_win[i] = sw[i];
    }
    c->apply_ola = apply_ola != 0;
    if (radix_pattern && radix_pattern_len > 0)
      c->radix_pattern.assign(radix_pattern, radix_pattern + radix_pattern_len);
    c->threads = threads > 0 ? threads : 1;
    c->lanes = lanes > 0 ? lanes : 1;
    c->has_pool = allow_outer_parallel != 0;
    c->logr_req = requested_logr(c);
    if (verbose()) {
      std::fprintf(stderr,
                   "[diag] fft_init_full: N=%d threads=%d lanes=%d allow_outer=%d allow_inner=%d "
                   "inner_threads=%d\n",
                   c->N, c->threads, c->lanes, allow_outer_parallel ? 1 : 0,
                   allow_inner_parallel ? 1 : 0, inner_threads);
    }
    try {
      setup_device(c);
    } catch (...) {
      delete c;
      return nullptr;
    }
    return c;
  } catch (...) {
    return nullptr;
  }
}

FFT_CFFI_API void* fft_init_full(size_t n, int threads, int lanes, int inverse, int kernel,
                                 int radix, const int* radix_pattern, size_t radix_pattern_len,
                                 int pad_mode, int window, int hop, int transform,
                                 int reduce_magnitude, int store_polar, int half_spectrum,
                                 int allow_outer_parallel, int allow_inner_parallel,
                                 int inner_threads, int save_crash_logs, int silent_crash_reports) {
  return fft_init_full_v2(n, threads, lanes, inverse, kernel, radix, radix_pattern,
                          radix_pattern_len, pad_mode, window, hop, transform, reduce_magnitude,
                          store_polar, half_spectrum, allow_outer_parallel, allow_inner_parallel,
                          inner_threads, save_crash_logs, silent_crash_reports, 0, 0, 0, 0.0f, 0.0f,
                          0, 0.0f, 0.0f, 0, 0);
}

FFT_CFFI_API void fft_free(void* handle) {
  FftContext* c = as_ctx(handle);
  if (!c) return;
  {
    DeviceGuard g(c->device);
    if (c->own_stream) {
      cudaStreamSynchronize(c->own_stream);
      cudaStreamDestroy(c->own_stream);
    }
    c->d_analysis.release();
    c->d_synthesis.release();
    c->d_weight.release();
    c->d_in0.release();
    c->d_in1.release();
    c->d_out0.release();
    c->d_out1.release();
    c->d_out2.release();
    c->d_frames.release();
    c->d_meta_tw.release();
    c->d_scratch.release();
    c->d_t2d.release();
    c->d_tma_timeouts.release();
    if (c->h_tma_timeouts) cudaFreeHost(c->h_tma_timeouts);
    c->d_gl_spec.release();
    c->d_gl_frames.release();
    c->d_gl_ola.release();
    c->d_gl_tmp.release();
    if (c->h_gl_cs) cudaFreeHost(c->h_gl_cs);
    for (cudaStream_t st : {c->up_stream, c->down_stream})
      if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
    for (cudaEvent_t e : c->pipe_events) cudaEventDestroy(e);
    c->magic = 0;
  }
  delete c;
}

FFT_CFFI_API void fft_pcm_to_channels(const float* in_pcm, float* out_real, float* out_imag,
                                      float* out_mag, size_t n, int threads) {
  // fft_cffi.cpp:431-513: forward C2C of the zero-padded signal (plan size the
  // next power of two), first n bins, |v| as magnitude.  Outputs are zeroed
  // on failure.
  (void)threads;
  if (!in_pcm || !out_real || !out_imag || !out_mag || n == 0) return;
  void* h = nullptr;
  try {
    const size_t plan_n = next_pow2(n);
    h = fft_init_full(plan_n, 1, 1, 0, 0, 0, nullptr, 0, 1, 0, 0, FFT_TRANSFORM_C2C, 0, 0, 0, 0, 0, 0,
                      0, 1);
    FftContext* c = as_ctx(h);
    if (!c) throw std::runtime_error("init");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    run_stft(c, in_pcm, n, 1, (int)n, (int)n, false, (int)n, false, PostFlags{}, false, out_real,
             out_imag, out_mag);
    fft_free(h);
  } catch (...) {
    if (h) fft_free(h);
    for (size_t i = 0; i < n; ++i) {
      out_real[i] = 0.f;
      out_imag[i] = 0.f;
      out_mag[i] = 0.f;
    }
  }
}

FFT_CFFI_API int fft_execute(void* handle, const float* in_pcm, float* out_real, float* out_imag,
                             float* out_mag, size_t n) {
  // fft_cffi.cpp:660-699
  FftContext* c = as_ctx(handle);
  if (!c || !in_pcm || !out_real || !out_imag || !out_mag || n == 0) return 0;
  if (c->pad_mode == 2 && (int)n != c->N) return 0;
  if (n > (size_t)c->N) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    run_stft(c, in_pcm, n, 1, (int)n, (int)n, false, c->N, false, c->post_flags(), stft_mirror(c),
             out_real, out_imag, out_mag);
    return 1;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API size_t fft_execute_batched(void* handle, const float* pcm, size_t pcm_len,
                                        float* out_real, float* out_imag, float* out_mag,
                                        int pad_mode, int enable_backup, size_t max_frames) {
  // fft_cffi.cpp:701-1034
  FftContext* c = as_ctx(handle);
  if (!c || !pcm || pcm_len == 0 || !out_real || !out_imag || !out_mag) return 0;
  const size_t frames = frame_count(c, pcm_len, pad_mode, max_frames);
  if (frames == 0) return 0;
  const int W = c->window ? c->window : c->N;
  const int H = c->hop ? c->hop : W;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    if (enable_backup && c->has_pool && c->allow_outer_parallel) {
      // Recovery path (fft_cffi.cpp:826-1027): the coordinator runs on the
      // host; frames it gives up on keep their restored, untransformed column.
      std::vector<char> raw;
      const size_t batch = recovery_batch_frames((size_t)c->N);
      run_stft(c, pcm, pcm_len, frames, W, H, true, c->bins(), true, c->post_flags(),
               stft_mirror(c), out_real, out_imag, out_mag);
      for (size_t b0 = 0; b0 < frames; b0 += batch) {
        const size_t cnt = std::min(batch, frames - b0);
        raw.assign(cnt, 0);
        run_recovery_coordinator(cnt, &raw);
        bool any = false;
        for (char r : raw) any = any || r;
        if (!any) continue;
        // Rewrite given-up frames with their framed input (re, 0, |re|).
        const int bins = c->bins();
        std::vector<float> seg(W), r_(bins), i_(bins, 0.f), m_(bins);
        for (size_t f = 0; f < cnt; ++f) {
          if (!raw[f]) continue;
          const size_t fi = b0 + f;
          const size_t start = fi * (size_t)H;
          size_t copy = 0;
          if (start < pcm_len) copy = std::min((size_t)W, pcm_len - start);
          if (copy) FFB_CHECK(cudaMemcpy(seg.data(), pcm + start, copy * 4, cudaMemcpyDefault));
          for (int k = 0; k < bins; ++k) {
            float v = 0.f;
            if ((size_t)k < copy) v = c->windows_enabled ? seg[k] * c->analysis_win[k] : seg[k];
            r_[k] = v;
            m_[k] = c->store_polar ? v : std::fabs(v);
          }
          FFB_CHECK(cudaMemcpy(out_real + fi * bins, r_.data(), bins * 4, cudaMemcpyDefault));
          FFB_CHECK(cudaMemcpy(out_imag + fi * bins, i_.data(), bins * 4, cudaMemcpyDefault));
          FFB_CHECK(cudaMemcpy(out_mag + fi * bins, m_.data(), bins * 4, cudaMemcpyDefault));
        }
      }
      return frames;
    }
    run_stft(c, pcm, pcm_len, frames, W, H, true, c->bins(), true, c->post_flags(), stft_mirror(c),
             out_real, out_imag, out_mag);
    return frames;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API size_t fft_stft_execute(void* handle, const float* pcm, size_t pcm_len,
                                     float* out_real, float* out_imag, float* out_mag,
                                     size_t max_frames) {
  return fft_execute_batched(handle, pcm, pcm_len, out_real, out_imag, out_mag, 1, 0, max_frames);
}

FFT_CFFI_API size_t fft_execute_complex_batched(void* handle, const float* in_real,
                                                const float* in_imag, size_t frames,
                                                float* out_pcm, int pad_mode, int enable_backup,
                                                size_t max_frames) {
  // fft_cffi.cpp:1042-1340
  (void)pad_mode;
  FftContext* c = as_ctx(handle);
  if (!c || !in_real || !in_imag || !out_pcm || frames == 0) return 0;
  if (c->N <= 0) return 0;
  if (max_frames != 0 && frames > max_frames) frames = max_frames;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    if (enable_backup && c->has_pool && c->allow_outer_parallel) {
      std::vector<char> raw(frames, 0);
      run_recovery_coordinator(frames, &raw);
      bool any = false;
      for (char r : raw) any = any || r;
      run_complex_batch(c, in_real, in_imag, frames, out_pcm, any ? &raw : nullptr);
      return frames;
    }
    run_complex_batch(c, in_real, in_imag, frames, out_pcm, nullptr);
    return frames;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API size_t fft_ctx_size(void* handle) {
  FftContext* c = as_ctx(handle);
  return c ? (size_t)c->N : 0;
}

FFT_CFFI_API size_t fft_ctx_worker_threads(void* handle) {
  // fft_cffi.cpp:1750-1759; the reference pool clamps to the hardware
  // thread count (eigen_fft.hpp:831-834).
  FftContext* c = as_ctx(handle);
  if (!c) return 0;
  if (c->has_pool) {
    int req = std::max(1, c->threads);
    const int hw = (int)std::thread::hardware_concurrency();
    if (hw > 0) req = std::min(req, hw);
    return (size_t)req;
  }
  return (size_t)(c->threads > 0 ? c->threads : 1);
}

FFT_CFFI_API size_t fft_ctx_effective_threads(void* handle) {
  // fft_cffi.cpp:1761-1773 -> Plan::effective_threads (eigen_fft.hpp:2332-2342)
  FftContext* c = as_ctx(handle);
  if (!c) return 0;
  int threads = c->threads > 0 ? c->threads : 4;
  threads = std::clamp(threads, 1, 16);
  int budget = threads;
  if (c->allow_inner_parallel) {
    int inner = c->inner_threads > 0 ? c->inner_threads : (int)std::thread::hardware_concurrency();
    inner = std::clamp(inner <= 0 ? 1 : inner, 1, 16);
    budget = std::max(budget, inner);
  }
  int hw = (int)std::thread::hardware_concurrency();
  if (hw <= 0) hw = 1;
  int eff = std::min(std::min(budget, hw), 16);
  return (size_t)std::max(1, eff);
}

FFT_CFFI_API int fft_config_window(void* handle, int analysis_kind, int synthesis_kind, float param1,
                                   float param2, int norm_policy, int cola_mode) {
  // fft_cffi.cpp:1983-2009: rebuilds length-W windows and leaves internal
  // window application disabled.
  FftContext* c = as_ctx(handle);
  if (!c) return 0;
  const int W = (c->window > 0) ? c->window : c->N;
  if (W <= 0) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->analysis_win_kind = analysis_kind;
    c->synthesis_win_kind = synthesis_kind;
    c->win_param1 = param1;
    c->win_param2 = param2;
    c->win_norm_policy = norm_policy;
    c->cola_mode = cola_mode;
    c->analysis_win = build_window(analysis_kind, W, param1, param2);
    c->synthesis_win = build_window(synthesis_kind, W, param1, param2);
    normalize_window(c->analysis_win, norm_policy);
    normalize_window(c->synthesis_win, norm_policy);
    c->windows_enabled = false;
    return 1;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API int fft_config_window_custom(void* handle, const float* analysis_window,
                                          size_t analysis_len, const float* synthesis_window,
                                          size_t synthesis_len, int norm_policy, int cola_mode) {
  // fft_cffi.cpp:2011-2032
  FftContext* c = as_ctx(handle);
  if (!c) return 0;
  const int W = (c->window > 0) ? c->window : c->N;
  if (W <= 0) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    if (analysis_window && analysis_len == (size_t)W)
      c->analysis_win.assign(analysis_window, analysis_window + analysis_len);
    if (synthesis_window && synthesis_len == (size_t)W)
      c->synthesis_win.assign(synthesis_window, synthesis_window + synthesis_len);
    c->win_norm_policy = norm_policy;
    c->cola_mode = cola_mode;
    normalize_window(c->analysis_win, norm_policy);
    normalize_window(c->synthesis_win, norm_policy);
    c->windows_enabled = false;
    return 1;
  } catch (...) {
    return 0;
  }
}

// ------------------------------------------------------------------ extensions
// The context's C2C plan flags over `batch` contiguous lines of N points.
static C2cArgs c2c_args(const FftContext* c, const float* in, float* out, size_t batch) {
  C2cArgs a{};
  a.in = reinterpret_cast<const float2*>(in);
  a.out = reinterpret_cast<float2*>(out);
  a.batch = (long long)batch;
  a.N = c->N;
  const int m = c->eff_transform();
  a.pre = c->stockham() ? 0 : (m == 1 ? 1 : ((m == 2 && c->half_spectrum) ? 2 : 0));
  a.polar_in = c->store_polar ? 1 : 0;
  a.inverse = c->inverse ? 1 : 0;
  a.pf = c->post_flags();
  return a;
}

// Contiguous lines: single pass, or the multi-pass kernels with the
// context's scratch.
static void run_c2c_lines(FftContext* c, const C2cArgs& a, cudaStream_t s) {
  if (single_pass(c->N, false)) {
    FFB_CHECK(launch_c2c(a, c->logr_req, s, &c->launches));
  } else {
    size_t chunk = 0;
    float2* scratch = scratch_for(c, c->N, a.batch, &chunk);
    FFB_CHECK(launch_four_step_c2c(a, scratch, chunk, s, &c->launches));
  }
}

FFT_CFFI_API int fftfree_execute_2d(void* ctx_axis0, void* ctx_axis1, const float* in, float* out, size_t rows,
                                    size_t cols, size_t batch) {
  // eigen_fft.hpp:3177-3215
  FftContext* c0 = as_ctx(ctx_axis0);
  FftContext* c1 = as_ctx(ctx_axis1);
  if (!c0 || !c1 || !in || !out || rows == 0 || cols == 0 || batch == 0) return 0;
  if ((size_t)c0->N != rows || (size_t)c1->N != cols) return 0;
  if (c0->device != c1->device) return 0;
  try {
    std::unique_lock<std::recursive_mutex> l0(c0->mu, std::defer_lock), l1(c1->mu, std::defer_lock);
    if (c0 == c1) {
      l0.lock();
    } else {
      std::lock(l0, l1);
    }
    DeviceGuard g(c0->device);
    cudaStream_t s = c0->stream;
    // an earlier asynchronous call whose TMA row pass gave up reports here
    if (c0->h_tma_timeouts && *(volatile unsigned*)c0->h_tma_timeouts) {
      FFB_CHECK(cudaStreamSynchronize(s));
      *c0->h_tma_timeouts = 0;
      FFB_CHECK(cudaMemsetAsync(c0->d_tma_timeouts.get(sizeof(unsigned)), 0, sizeof(unsigned), s));
      if (verbose()) std::fprintf(stderr, "[fftfree_b200] an earlier 2-D call's row pass gave up waiting\n");
      return 0;
    }
    const size_t n = batch * rows * cols * 2;
    const bool in_host = !is_device_ptr(in);
    OutTarget o = stage_out(c0->d_out0, out, n);
    const float* d_in = stage_in(c0, c0->d_in0, in, n);
    // axis 0: the columns are contiguous lines of `rows` points
    run_c2c_lines(c0, c2c_args(c0, d_in, o.dev, batch * cols), s);
    // axis 1: row r of matrix m is the line of `cols` points r + j * rows
    C2cArgs a1 = c2c_args(c1, o.dev, o.dev, batch * rows);
    bool tma_check = false;
    if (ilog2(cols) <= max_strided_log()) {
      StridedLinesArgs sl{a1, (long long)rows};
      sl.timeouts = static_cast<unsigned*>(c0->d_tma_timeouts.get(sizeof(unsigned)));
      if (!c0->h_tma_timeouts) {
        FFB_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&c0->h_tma_timeouts), sizeof(unsigned),
                                cudaHostAllocDefault));
        *c0->h_tma_timeouts = 0;
        FFB_CHECK(cudaMemsetAsync(sl.timeouts, 0, sizeof(unsigned), s));
      }
      FFB_CHECK(launch_c2c_strided(sl, c1->logr_req, s, &c1->launches));
      FFB_CHECK(cudaMemcpyAsync(c0->h_tma_timeouts, sl.timeouts, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
      tma_check = true;
    } else {
      // lines beyond one pass: transpose, multi-pass over contiguous rows,
      // transpose back (the reference's own route)
      float2* t = static_cast<float2*>(c0->d_t2d.get(n * sizeof(float)));
      float2* d = reinterpret_cast<float2*>(o.dev);
      FFB_CHECK(launch_transpose(d, t, (long long)rows, (long long)cols, (long long)batch, s, &c0->launches));
      a1.in = t;
      a1.out = t;
      size_t chunk = 0;
      float2* scratch = scratch_for(c1, c1->N, a1.batch, &chunk);
      FFB_CHECK(launch_four_step_c2c(a1, scratch, chunk, s, &c1->launches));
      FFB_CHECK(launch_transpose(t, d, (long long)cols, (long long)rows, (long long)batch, s, &c0->launches));
    }
    finish_out(c0, o);
    finish_call(c0, in_host || o.host);
    if (tma_check && (in_host || o.host || !c0->async) && *c0->h_tma_timeouts) {
      // the call synchronised, so its count is here: a block gave up
      *c0->h_tma_timeouts = 0;
      FFB_CHECK(cudaMemsetAsync(c0->d_tma_timeouts.get(sizeof(unsigned)), 0, sizeof(unsigned), s));
      FFB_CHECK(cudaStreamSynchronize(s));
      if (verbose()) std::fprintf(stderr, "[fftfree_b200] 2-D row pass: a bounded wait gave up\n");
      return 0;
    }
    return 1;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API int fftfree_execute_c2c(void* handle, const float* in, float* out, size_t batch) {
  FftContext* c = as_ctx(handle);
  if (!c || !in || !out || batch == 0) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const size_t n = batch * (size_t)c->N * 2;
    const bool in_host = !is_device_ptr(in);
    OutTarget o = stage_out(c->d_out0, out, n);
    const bool any_host = in_host || o.host;
    const int chunks = single_pass(c->N, false)
                           ? pipe_chunks(n * 4 * ((in_host ? 1 : 0) + (o.host ? 1 : 0)), (long long)batch)
                           : 1;
    const float* d_in = (chunks > 1 && in_host) ? static_cast<const float*>(c->d_in0.get(n * sizeof(float)))
                                                : stage_in(c, c->d_in0, in, n);
    C2cArgs a = c2c_args(c, d_in, o.dev, batch);
    if (chunks > 1) {
      const size_t per = (batch + chunks - 1) / chunks, row = (size_t)c->N * 2;
      auto rows = [&](int i, size_t* r0, size_t* r1) {
        *r0 = std::min(batch, (size_t)i * per);
        *r1 = std::min(batch, *r0 + per);
      };
      run_pipelined(
          c, chunks,
          [&](int i, cudaStream_t s) {
            size_t r0, r1;
            rows(i, &r0, &r1);
            if (in_host) copy_h2d(const_cast<float*>(d_in) + r0 * row, in + r0 * row, (r1 - r0) * row, s);
          },
          [&](int i, cudaStream_t s) {
            size_t r0, r1;
            rows(i, &r0, &r1);
            if (r1 <= r0) return;
            C2cArgs b = a;
            b.in = a.in + r0 * (size_t)c->N;
            b.out = a.out + r0 * (size_t)c->N;
            b.batch = (long long)(r1 - r0);
            FFB_CHECK(launch_c2c(b, c->logr_req, s, &c->launches));
          },
          [&](int i, cudaStream_t s) {
            size_t r0, r1;
            rows(i, &r0, &r1);
            if (o.host) copy_d2h(o.user + r0 * row, o.dev + r0 * row, (r1 - r0) * row, s);
          });
      finish_call(c, true);
      return 1;
    }
    run_c2c_lines(c, a, c->stream);
    finish_out(c, o);
    finish_call(c, any_host);
    return 1;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API int fftfree_execute_c2c_meta(void* handle, const float* in, float* out, size_t batch,
                                          const fftfree_metadata_request* requests, int request_count) {
  FftContext* c = as_ctx(handle);
  if (!c || !in || !out || batch == 0) return 0;
  if (request_count > 0 && !requests) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    return run_meta(c, in, out, batch, requests, request_count);
  } catch (...) {
    return 0;
  }
}

// ------------------------------------------------------------------ gradients
// Magnitude STFT of `signals` signals (row stride `length`) and its
// gradient; the context fixes N, window, hop, pad rule and analysis window.
static bool mag_grad_ctx_ok(const FftContext* c, const char* who) {
  const bool ok = !c->inverse && c->eff_transform() == FFT_TRANSFORM_R2C && c->half_spectrum &&
                  c->N >= 2 && ilog2((size_t)c->N) <= max_mag_grad_log();
  if (!ok)
    std::fprintf(stderr, "[fftfree_b200] %s: needs a forward R2C half-spectrum context with 2 <= N <= %d\n",
                 who, 1 << max_mag_grad_log());
  return ok;
}

static int mag_grad_span(int H) {
  static const int env = [] {
    const char* e = std::getenv("FFTFREE_GRAD_SPAN");
    return e ? std::atoi(e) : 0;
  }();
  if (env > 0) return env;
  // about 16 hops of one signal per block, at least one hop
  long long s = 16LL * H;
  if (s > 8192) s = std::max(8192, H);
  return (int)s;
}

static int mag_grad_run() {
  static const int env = [] {
    const char* e = std::getenv("FFTFREE_GRAD_RUN");
    return e ? std::atoi(e) : -1;
  }();
  // frames per thread group (FFTFREE_GRAD_RUN, for sweeps); 0 selects the
  // general form, -1 lets the launcher fit the runs to the GPU
  return env >= 0 ? env : -1;
}

// Shared body of the magnitude STFT entry points; out_phasor (X / |X| as
// interleaved pairs, 0 where |X| = 0) is written when not null; with a
// target, out_mag receives |X| - target and out_partials the squared
// residuals' partial sums.
static size_t stft_magnitude(void* handle, const float* pcm, size_t signals, size_t length, float* out_mag,
                             float* out_phasor, size_t max_frames, const char* who, const float* target = nullptr,
                             float* out_partials = nullptr) {
  FftContext* c = as_ctx(handle);
  if (!c || !pcm || !out_mag || signals == 0 || length == 0) return 0;
  if (target && (!out_phasor || !out_partials)) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    if (!mag_grad_ctx_ok(c, who)) return 0;
    DeviceGuard g(c->device);
    const size_t frames = frame_count(c, length, 0, max_frames);
    if (frames == 0) return 0;
    const int W = c->window ? c->window : c->N;
    const int H = c->hop ? c->hop : W;
    const int bins = c->N / 2 + 1;
    const size_t outn = signals * frames * (size_t)bins;
    bool any_host = !is_device_ptr(pcm);
    const float* d_pcm = stage_in(c, c->d_in0, pcm, signals * length);
    OutTarget o = stage_out(c->d_out2, out_mag, outn);
    OutTarget op, opart;
    if (out_phasor) op = stage_out(c->d_out1, out_phasor, 2 * outn);
    const float* d_tg = nullptr;
    const long long nparts = stft_loss_parts((long long)(signals * frames), c->N);
    if (target) {
      any_host = any_host || !is_device_ptr(target);
      d_tg = stage_in(c, c->d_in1, target, outn);
      opart = stage_out(c->d_frames, out_partials, (size_t)nparts);
    }
    any_host = any_host || o.host || op.host || opart.host;
    StftArgs a{};
    a.pcm = d_pcm;
    a.pcm_len = (long long)length;
    a.frames = (long long)(signals * frames);
    a.N = c->N;
    a.W = W;
    a.H = H;
    a.win = c->windows_enabled ? static_cast<const float*>(c->d_analysis.p) : nullptr;
    a.pf = c->post_flags();
    a.out_bins = bins;
    a.out_stride = bins;
    a.out_mag = o.dev;
    a.out_phasor = out_phasor ? reinterpret_cast<float2*>(op.dev) : nullptr;
    a.sig_frames = (long long)frames;
    a.sig_stride = (long long)length;
    a.mag_only = target ? 3 : (out_phasor ? 2 : 1);
    a.target = d_tg;
    a.loss_part = target ? opart.dev : nullptr;
    FFB_CHECK(launch_stft(a, c->logr_req, c->stream, &c->launches));
    finish_out(c, o);
    if (out_phasor) finish_out(c, op);
    if (target) finish_out(c, opart);
    finish_call(c, any_host);
    return frames;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API size_t fftfree_stft_magnitude(void* handle, const float* pcm, size_t signals, size_t length,
                                           float* out_mag, size_t max_frames) {
  return stft_magnitude(handle, pcm, signals, length, out_mag, nullptr, max_frames, "fftfree_stft_magnitude");
}

FFT_CFFI_API size_t fftfree_stft_magnitude_phasor(void* handle, const float* pcm, size_t signals, size_t length,
                                                  float* out_mag, float* out_phasor, size_t max_frames) {
  if (!out_phasor) return 0;
  return stft_magnitude(handle, pcm, signals, length, out_mag, out_phasor, max_frames,
                        "fftfree_stft_magnitude_phasor");
}

FFT_CFFI_API size_t fftfree_stft_l2_partials(void* handle, size_t frames_total) {
  FftContext* c = as_ctx(handle);
  return c ? (size_t)stft_loss_parts((long long)frames_total, c->N) : 0;
}

FFT_CFFI_API size_t fftfree_stft_magnitude_l2(void* handle, const float* pcm, size_t signals, size_t length,
                                              const float* target, float* out_residual, float* out_phasor,
                                              float* out_partials, size_t max_frames) {
  if (!target || !out_phasor || !out_partials) return 0;
  return stft_magnitude(handle, pcm, signals, length, out_residual, out_phasor, max_frames,
                        "fftfree_stft_magnitude_l2", target, out_partials);
}

// Shared body of the gradient entry points: the spectrum comes from pcm
// (recomputed) or from a saved unit phasor.
static size_t stft_magnitude_backward(void* handle, const float* pcm, const float* phasor, size_t signals,
                                      size_t length, const float* grad_mag, float* grad_pcm, const char* who,
                                      const float* scale = nullptr, float factor = 1.0f) {
  FftContext* c = as_ctx(handle);
  if (!c || !(pcm || phasor) || !grad_mag || !grad_pcm || signals == 0 || length == 0) return 0;
  try {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    if (!mag_grad_ctx_ok(c, who)) return 0;
    DeviceGuard g(c->device);
    const size_t frames = frame_count(c, length, 0, 0);
    if (frames == 0) return 0;
    const int W = c->window ? c->window : c->N;
    const int H = c->hop ? c->hop : W;
    const int bins = c->N / 2 + 1;
    const size_t specn = signals * frames * (size_t)bins;
    bool any_host = !is_device_ptr(grad_mag);
    const float* d_pcm = nullptr;
    const float* d_ph = nullptr;
    if (phasor) {
      any_host = any_host || !is_device_ptr(phasor);
      d_ph = stage_in(c, c->d_in0, phasor, 2 * specn);
    } else {
      any_host = any_host || !is_device_ptr(pcm);
      d_pcm = stage_in(c, c->d_in0, pcm, signals * length);
    }
    const float* d_g = stage_in(c, c->d_in1, grad_mag, specn);
    OutTarget o = stage_out(c->d_out0, grad_pcm, signals * length);
    any_host = any_host || o.host;
    MagGradArgs a{};
    a.pcm = d_pcm;
    a.phasor = reinterpret_cast<const float2*>(d_ph);
    a.signals = (long long)signals;
    a.pcm_len = (long long)length;
    a.sig_stride = (long long)length;
    a.frames = (long long)frames;
    a.N = c->N;
    a.W = W;
    a.H = H;
    a.win = c->windows_enabled ? static_cast<const float*>(c->d_analysis.p) : nullptr;
    a.grad_mag = d_g;
    a.grad_pcm = o.dev;
    a.span = mag_grad_span(H);
    a.run = mag_grad_run();
    a.factor = factor;
    a.scale = scale;
    if (scale && !is_device_ptr(scale)) throw std::runtime_error("scale must be device memory");
    FFB_CHECK(launch_stft_mag_grad(a, c->logr_req, c->stream, &c->launches));
    finish_out(c, o);
    finish_call(c, any_host);
    return frames;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API size_t fftfree_stft_magnitude_backward(void* handle, const float* pcm, size_t signals,
                                                    size_t length, const float* grad_mag, float* grad_pcm) {
  if (!pcm) return 0;
  return stft_magnitude_backward(handle, pcm, nullptr, signals, length, grad_mag, grad_pcm,
                                 "fftfree_stft_magnitude_backward");
}

FFT_CFFI_API size_t fftfree_stft_magnitude_backward_phasor(void* handle, const float* phasor, size_t signals,
                                                           size_t length, const float* grad_mag,
                                                           float* grad_pcm) {
  if (!phasor) return 0;
  return stft_magnitude_backward(handle, nullptr, phasor, signals, length, grad_mag, grad_pcm,
                                 "fftfree_stft_magnitude_backward_phasor");
}

FFT_CFFI_API size_t fftfree_stft_magnitude_backward_phasor_scaled(void* handle, const float* phasor,
                                                                  size_t signals, size_t length,
                                                                  const float* grad_mag, float* grad_pcm,
                                                                  const float* scale, float factor) {
  if (!phasor) return 0;
  return stft_magnitude_backward(handle, nullptr, phasor, signals, length, grad_mag, grad_pcm,
                                 "fftfree_stft_magnitude_backward_phasor_scaled", scale, factor);
}

FFT_CFFI_API void fftfree_set_stream(void* handle, void* cuda_stream) {
  FftContext* c = as_ctx(handle);
  if (!c) return;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->stream = static_cast<cudaStream_t>(cuda_stream);
}

FFT_CFFI_API void* fftfree_ctx_stream(void* handle) {
  FftContext* c = as_ctx(handle);
  return c ? static_cast<void*>(c->stream) : nullptr;
}

FFT_CFFI_API void fftfree_set_async(void* handle, int on) {
  FftContext* c = as_ctx(handle);
  if (!c) return;
  c->async = on != 0;
}

FFT_CFFI_API unsigned long long fftfree_ctx_launch_count(void* handle) {
  FftContext* c = as_ctx(handle);
  return c ? (unsigned long long)c->launches : 0ull;
}

FFT_CFFI_API size_t fftfree_frame_count(void* handle, size_t pcm_len, int pad_mode, size_t max_frames) {
  FftContext* c = as_ctx(handle);
  return c ? frame_count(c, pcm_len, pad_mode, max_frames) : 0;
}

FFT_CFFI_API int fftfree_ctx_frame_shape(void* handle, int* window, int* hop) {
  FftContext* c = as_ctx(handle);
  if (!c) return 0;
  const int W = c->window ? c->window : c->N;
  const int H = c->hop ? c->hop : W;
  if (window) *window = W;
  if (hop) *hop = H;
  return 1;
}

FFT_CFFI_API int fftfree_ctx_kernel(void* handle) {
  FftContext* c = as_ctx(handle);
  return c ? c->kernel : -1;
}

FFT_CFFI_API int fftfree_ctx_schedule(void* handle, int* radices, int max_passes) {
  FftContext* c = as_ctx(handle);
  if (!c || !radices || max_passes <= 0) return 0;
  const int lg = ilog2((size_t)c->N);
  const bool real_in = c->eff_transform() == 1;  // batched STFT of real frames halves the size
  const int logm = real_in ? std::max(0, lg - 1) : lg;
  const int logr = choose_logr(logm, c->logr_req, real_in);
  if (logr < 0) return 0;
  const int lr = std::min(logr, logm);
  int n = 0;
  if (lr > 0 && logm % lr) radices[n++] = 1 << (logm % lr);
  for (int p = 0; lr > 0 && p < logm / lr && n < max_passes; ++p) radices[n++] = 1 << lr;
  return n;
}

}  // extern "C"
