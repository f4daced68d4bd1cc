// stream.cpp -- streaming STFT/ISTFT buffers, Griffin-Lim and phase
// inference: the reference's host-side drivers over the batched entry points
// (fft_cffi.cpp:1342-1742, 2058-2248; phase_infer.hpp).  Every transform they
// issue runs through the GPU entry points of abi.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <stdexcept>
#include <vector>

#include "../../include/fft_cffi.h"
#include "../../include/fftfree_b200.h"
#include "context.h"
#include "kernels.h"

namespace ffb {
namespace {

bool verbose() {
  static const bool v = [] {
    const char* e = std::getenv("FFTFREE_VERBOSE");
    return e && *e && e[0] != '0';
  }();
  return v;
}

int stream_window(const FftContext* c) { return c->window > 0 ? c->window : c->N; }
int stream_hop(const FftContext* c) { return c->hop > 0 ? c->hop : stream_window(c); }

size_t stream_backlog(const FftContext* c) {
  if (c->streaming_offset >= c->streaming_buffer.size()) return 0;
  return c->streaming_buffer.size() - c->streaming_offset;
}

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

void stream_compact(FftContext* c) {
  if (c->streaming_offset == 0) return;
  if (c->streaming_offset >= c->streaming_buffer.size()) {
    c->streaming_buffer.clear();
    c->streaming_offset = 0;
    return;
  }
  c->streaming_buffer.erase(c->streaming_buffer.begin(),
                            c->streaming_buffer.begin() + (std::ptrdiff_t)c->streaming_offset);
  c->streaming_offset = 0;
}

size_t stream_inverse_pending(const FftContext* c) {
  if (c->streaming_inverse_queue.empty()) return 0;
  if (c->streaming_inverse_offset >= c->streaming_inverse_queue.size()) return 0;
  return c->streaming_inverse_queue.size() - c->streaming_inverse_offset;
}

void stream_inverse_compact(FftContext* c) {
  if (c->streaming_inverse_offset == 0) return;
  if (c->streaming_inverse_offset >= c->streaming_inverse_queue.size()) {
    c->streaming_inverse_queue.clear();
    c->streaming_inverse_offset = 0;
    return;
  }
  c->streaming_inverse_queue.erase(
      c->streaming_inverse_queue.begin(),
      c->streaming_inverse_queue.begin() + (std::ptrdiff_t)c->streaming_inverse_offset);
  c->streaming_inverse_offset = 0;
}

size_t stream_inverse_emit(FftContext* c, float* out_pcm, size_t max_samples) {
  const size_t pending = stream_inverse_pending(c);
  if (pending == 0) return 0;
  size_t take = pending;
  if (max_samples != 0 && take > max_samples) take = max_samples;
  if (!out_pcm || take == 0) return 0;
  std::copy_n(c->streaming_inverse_queue.data() + c->streaming_inverse_offset, take, out_pcm);
  c->streaming_inverse_offset += take;
  stream_inverse_compact(c);
  return take;
}

float cola_weight(const FftContext* c, size_t i) {
  if (!c->windows_enabled) return 1.0f;
  const float a = (i < c->analysis_win.size()) ? c->analysis_win[i] : 1.0f;
  const float s = (i < c->synthesis_win.size()) ? c->synthesis_win[i] : 1.0f;
  return a * s;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" {

FFT_CFFI_API void fft_stream_reset(void* handle) {
  FftContext* c = as_ctx(handle);
  if (!c) return;
  c->streaming_buffer.clear();
  c->streaming_offset = 0;
  c->streaming_inverse_queue.clear();
  c->streaming_inverse_offset = 0;
  c->streaming_inverse_accum.clear();
  c->streaming_inverse_norm.clear();
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
  return stream_inverse_pending(c);
}

FFT_CFFI_API size_t fft_stream_push_pcm(void* handle, const float* pcm, size_t samples,
                                        float* out_real, float* out_imag, float* out_mag,
                                        size_t max_frames, int flush_mode) {
  // fft_cffi.cpp:1508-1595.  The reference prints a diagnostic line on every
  // call; here that needs FFTFREE_VERBOSE.
  (void)flush_mode;
  FftContext* c = as_ctx(handle);
  if (!c) {
    if (verbose()) std::fprintf(stderr, "[fft_stream_push_pcm] handle is NULL\n");
    return 0;
  }
  if (samples > 0 && pcm) c->streaming_buffer.insert(c->streaming_buffer.end(), pcm, pcm + samples);
  const int W = stream_window(c), H = stream_hop(c);
  if (verbose())
    std::fprintf(stderr, "[fft_stream_push_pcm] samples=%zu W=%d H=%d offset=%zu buf_size=%zu\n",
                 samples, W, H, c->streaming_offset, c->streaming_buffer.size());
  if (W <= 0 || H <= 0) return 0;
  const size_t backlog = stream_backlog(c);
  const size_t available = stream_available_frames(c);
  if (available == 0) return 0;
  size_t frames = available;
  if (max_frames != 0 && frames > max_frames) frames = max_frames;
  size_t pcm_len = (size_t)W + (frames - 1) * (size_t)H;
  if (pcm_len > backlog) pcm_len = backlog;
  std::vector<float> chunk(pcm_len, 0.0f);
  for (size_t f = 0; f < frames; ++f) {
    const size_t fs = f * (size_t)H;
    const size_t src = c->streaming_offset + fs;
    for (int wi = 0; wi < W; ++wi) {
      const size_t ci = fs + (size_t)wi;
      if (ci >= chunk.size()) break;
      float v = 0.0f;
      if (src + (size_t)wi < c->streaming_buffer.size()) v = c->streaming_buffer[src + (size_t)wi];
      chunk[ci] = v;
    }
  }
  const size_t bins = stream_bins(c);
  std::vector<float> lr(out_real ? 0 : frames * bins), li(out_imag ? 0 : frames * bins),
      lm(out_mag ? 0 : frames * bins);
  float* rt = out_real ? out_real : lr.data();
  float* it = out_imag ? out_imag : li.data();
  float* mt = out_mag ? out_mag : lm.data();
  const size_t produced = fft_execute_batched(handle, chunk.data(), pcm_len, rt, it, mt, 2, 0, frames);
  if (produced == 0) return 0;
  c->streaming_offset += produced * (size_t)H;
  stream_compact(c);
  return produced;
}

FFT_CFFI_API size_t fft_stream_push_spectrum(void* handle, const float* in_real,
                                             const float* in_imag, size_t frames, float* out_pcm,
                                             size_t max_samples, int flush_mode) {
  // fft_cffi.cpp:1597-1742
  FftContext* c = as_ctx(handle);
  if (!c || !c->inverse) return 0;
  const size_t plan_n = (size_t)std::max(c->N, 1);
  const size_t bins = stream_bins(c);
  if (c->streaming_inverse_accum.size() != plan_n) c->streaming_inverse_accum.assign(plan_n, 0.0f);
  const bool use_norm = (c->cola_mode == FFT_COLA_NORMALIZE);
  if (use_norm) {
    if (c->streaming_inverse_norm.size() != plan_n) c->streaming_inverse_norm.assign(plan_n, 0.0f);
  } else {
    c->streaming_inverse_norm.clear();
  }
  if (frames > 0) {
    if (!in_real) return stream_inverse_emit(c, out_pcm, max_samples);
    const size_t total_bins = frames * bins;
    std::vector<float> tr(in_real, in_real + total_bins);
    std::vector<float> ti;
    const float* imag_ptr = nullptr;
    if (in_imag) {
      ti.assign(in_imag, in_imag + total_bins);
      imag_ptr = ti.data();
    }
    std::vector<float> frame_pcm(frames * plan_n, 0.0f);
    // A NULL imaginary part fails the batch (as in the reference), which then
    // only drains what is queued.
    size_t produced = fft_execute_complex_batched(handle, tr.data(), imag_ptr, frames,
                                                  frame_pcm.data(), 2, 0, frames);
    if (produced == 0) return stream_inverse_emit(c, out_pcm, max_samples);
    if (produced > frames) produced = frames;
    const size_t hop = (size_t)std::max(stream_hop(c), 1);
    for (size_t f = 0; f < produced; ++f) {
      const float* fr = frame_pcm.data() + f * plan_n;
      for (size_t i = 0; i < plan_n; ++i) {
        c->streaming_inverse_accum[i] += fr[i];
        if (use_norm) c->streaming_inverse_norm[i] += cola_weight(c, i);
      }
      size_t emit = hop;
      if (flush_mode == FFT_STREAM_FLUSH_FINAL && (f + 1 == produced)) emit = plan_n;
      if (emit > plan_n) emit = plan_n;
      for (size_t i = 0; i < emit; ++i) {
        float s = c->streaming_inverse_accum[i];
        if (use_norm) {
          const float d = c->streaming_inverse_norm[i];
          if (std::fabs(d) > 1e-12f) s /= d;
        }
        c->streaming_inverse_queue.push_back(s);
      }
      if (emit < plan_n) {
        std::move(c->streaming_inverse_accum.begin() + emit, c->streaming_inverse_accum.end(),
                  c->streaming_inverse_accum.begin());
        std::fill(c->streaming_inverse_accum.end() - emit, c->streaming_inverse_accum.end(), 0.0f);
        if (use_norm) {
          std::move(c->streaming_inverse_norm.begin() + emit, c->streaming_inverse_norm.end(),
                    c->streaming_inverse_norm.begin());
          std::fill(c->streaming_inverse_norm.end() - emit, c->streaming_inverse_norm.end(), 0.0f);
        }
      } else {
        std::fill(c->streaming_inverse_accum.begin(), c->streaming_inverse_accum.end(), 0.0f);
        if (use_norm) std::fill(c->streaming_inverse_norm.begin(), c->streaming_inverse_norm.end(), 0.0f);
      }
    }
  }
  if (flush_mode == FFT_STREAM_FLUSH_FINAL && frames == 0) {
    if (!c->streaming_inverse_accum.empty()) {
      const bool nl = !c->streaming_inverse_norm.empty();
      for (size_t i = 0; i < c->streaming_inverse_accum.size(); ++i) {
        float s = c->streaming_inverse_accum[i];
        if (nl) {
          const float d = c->streaming_inverse_norm[i];
          if (std::fabs(d) > 1e-12f) s /= d;
        }
        c->streaming_inverse_queue.push_back(s);
      }
      std::fill(c->streaming_inverse_accum.begin(), c->streaming_inverse_accum.end(), 0.0f);
      if (nl) std::fill(c->streaming_inverse_norm.begin(), c->streaming_inverse_norm.end(), 0.0f);
    }
  }
  return stream_inverse_emit(c, out_pcm, max_samples);
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
    // std::mt19937 and a float uniform in [-pi, pi), on the host.
    const float kPi = 3.14159265358979323846f;
    std::mt19937 rng(seed ? seed : 0x47d7bfad);
    std::uniform_real_distribution<float> dist(-kPi, kPi);
    // A device-resident magnitude is read back once for the initial spectra.
    std::vector<float> mag_host;
    const float* hmag = in_mag;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, in_mag) == cudaSuccess && pa.type == cudaMemoryTypeDevice) {
      mag_host.resize(total_bins);
      if (cudaMemcpy(mag_host.data(), in_mag, total_bins * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return 0;
      hmag = mag_host.data();
    } else {
      cudaGetLastError();
    }
    std::vector<float> re0(total_bins), im0(total_bins);
    for (size_t i = 0; i < total_bins; ++i) {
      const float a = dist(rng);
      re0[i] = hmag[i] * std::cos(a);
      im0[i] = hmag[i] * std::sin(a);
    }
    // The iterations run on the device (phase_infer.hpp:140-208): the inverse
    // batch, the count-normalised overlap-add, the forward STFT and the phase
    // projection, with every intermediate in device memory.
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != fc->device) cudaSetDevice(fc->device);
    struct Restore {
      int dev;
      ~Restore() {
        if (dev >= 0) cudaSetDevice(dev);
      }
    } restore{prev != fc->device ? prev : -1};
    DevBuf d_mag, d_re, d_im, d_frames, d_ola, d_tr, d_ti, d_tm;
    const size_t fb = total_bins * sizeof(float);
    float* mag = static_cast<float*>(d_mag.get(fb));
    float* re = static_cast<float*>(d_re.get(fb));
    float* im = static_cast<float*>(d_im.get(fb));
    float* tr = static_cast<float*>(d_tr.get(fb));
    float* ti = static_cast<float*>(d_ti.get(fb));
    float* tm = static_cast<float*>(d_tm.get(fb));
    float* frame_pcm = static_cast<float*>(d_frames.get(frames * plan_n * sizeof(float)));
    const size_t ola_cap = std::max(ola_len, frames * plan_n);
    float* ola = static_cast<float*>(d_ola.get(ola_cap * sizeof(float)));
    cudaStream_t st = fc->stream;
    auto ok = [](cudaError_t e) {
      if (e != cudaSuccess) throw std::runtime_error("cuda");
    };
    ok(cudaMemcpyAsync(mag, in_mag, fb, cudaMemcpyDefault, st));
    ok(cudaMemcpyAsync(re, re0.data(), fb, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(im, im0.data(), fb, cudaMemcpyHostToDevice, st));
    ok(cudaStreamSynchronize(st));
    // The reference refines out_real/out_imag in place, so a failed pass
    // leaves the spectra of the last completed one there.
    auto flush = [&]() {
      ok(cudaMemcpyAsync(out_real, re, fb, cudaMemcpyDefault, st));
      ok(cudaMemcpyAsync(out_imag, im, fb, cudaMemcpyDefault, st));
      ok(cudaStreamSynchronize(st));
    };
    for (int it = 0; it < iters; ++it) {
      const size_t pr = fft_execute_complex_batched(ctx_inverse, re, im, frames, frame_pcm, pad_mode, 0, frames);
      if (pr == 0) {
        flush();
        return 0;
      }
      ok(cudaStreamSynchronize(ic->stream));
      const size_t uf = std::min(pr, frames);
      ok(cudaMemsetAsync(ola, 0, ola_cap * sizeof(float), st));
      OlaArgs o{};
      o.frames_buf = frame_pcm;
      o.frames = (long long)uf;
      o.N = (int)plan_n;
      o.H = (int)hp;
      o.cola = 1;  // divide by the number of frames covering the sample
      o.weight = nullptr;
      o.out = ola;
      ok(launch_ola(o, st, &fc->launches));
      ok(cudaStreamSynchronize(st));
      const size_t ff = fft_execute_batched(ctx_forward, ola, ola_len, tr, ti, tm, pad_mode, 0, frames);
      if (ff == 0) {
        flush();
        return 0;
      }
      ok(cudaStreamSynchronize(fc->stream));
      const size_t uff = std::min(ff, frames);
      ok(launch_gl_project(mag, tr, ti, re, im, (long long)(uff * bins), (int)bins, half ? 1 : 0,
                           (plan_n & 1) == 0 ? 1 : 0, st));
      ok(cudaStreamSynchronize(st));
    }
    flush();
    return 1;
  } catch (...) {
    return 0;
  }
}

}  // extern "C"
