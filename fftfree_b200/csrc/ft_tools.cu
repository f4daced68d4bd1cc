// ft_tools.cu -- the spectrogram-grid pipeline (ft_tools.hpp:145-481 behind
// ft_tools_cffi.cpp:76-174) on the GPU: the step after the STFT that
// resamples, quantizes and contrast-boosts a time x freq grid.
//
// Every unit is one launch over the grid (row-major, freq fastest: each warp
// reads and writes whole rows, coalesced): bilinear upsampling gathers its
// four corners, the quantizer and the contrast update are per cell, the local
// mean of the contrast booster is a window sum read through L1 (or, when a
// window spans a whole axis, column / row sums in FP64 made once), and box
// downsampling sums its cells.  Floating-point steps follow the reference's
// order with rounded (non-contracted) products; the transcendental functions
// are CUDA's (hypot, atan2, sin / cos, exp, pow), within a few ulp of the
// host's.  Polar grids go through complex values exactly where the reference
// converts them (resampling), and stay magnitude-only elsewhere.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <mutex>
#include <stdexcept>

#include "../../include/ft_tools_cffi.h"
#include "context.h"

namespace ffb {
namespace {

struct QuantP {
  float base_frequency, magnitude_step, mix, distance_decay;
};
struct ContrastP {
  float brightness, contrast, gamma;
  int clamp_zero;
};

__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
  return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), t));  // a + (b - a) * t
}
__device__ __forceinline__ float2 lerp_c(float2 a, float2 b, float t) {
  return make_float2(lerp_rn(a.x, b.x, t), lerp_rn(a.y, b.y, t));
}
__device__ __forceinline__ float2 polar_c(float m, float ph) {  // std::polar
  float s, c;
  sincosf(ph, &s, &c);
  return make_float2(__fmul_rn(m, c), __fmul_rn(m, s));
}
__device__ __forceinline__ float cabs_c(float2 v) { return hypotf(v.x, v.y); }  // std::abs
__device__ __forceinline__ float carg_c(float2 v) { return atan2f(v.y, v.x); }  // std::arg

// element of a planar grid as a complex value (polar grids converted)
template <bool POLAR>
__device__ __forceinline__ float2 load_c(const float* a0, const float* a1, long long i) {
  const float x = __ldg(a0 + i), y = __ldg(a1 + i);
  return POLAR ? polar_c(x, y) : make_float2(x, y);
}
template <bool POLAR>
__device__ __forceinline__ void store_c(float* a0, float* a1, long long i, float2 v) {
  if (POLAR) {
    a0[i] = cabs_c(v);
    a1[i] = carg_c(v);
  } else {
    a0[i] = v.x;
    a1[i] = v.y;
  }
}

// ft_tools.hpp:145-179 (upsample_complex; polar grids via :219-227)
template <bool POLAR>
__global__ void k_ft_upsample(const float* __restrict__ s0, const float* __restrict__ s1, float* __restrict__ d0,
                              float* __restrict__ d1, int T, int F, int ut, int uf) {
  const int DT = T * ut, DF = F * uf;
  const long long total = (long long)DT * DF;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / DF), f = (int)(i - (long long)t * DF);
    const double st = (double)t / (double)ut, sf = (double)f / (double)uf;
    const int t0 = (int)floor(st), f0 = (int)floor(sf);
    const int t1 = min(t0 + 1, T - 1), f1 = min(f0 + 1, F - 1);
    const float tw = (float)(st - (double)t0), fw = (float)(sf - (double)f0);
    const float2 c00 = load_c<POLAR>(s0, s1, (long long)t0 * F + f0);
    const float2 c10 = load_c<POLAR>(s0, s1, (long long)t1 * F + f0);
    const float2 c01 = load_c<POLAR>(s0, s1, (long long)t0 * F + f1);
    const float2 c11 = load_c<POLAR>(s0, s1, (long long)t1 * F + f1);
    store_c<POLAR>(d0, d1, i, lerp_c(lerp_c(c00, c10, tw), lerp_c(c01, c11, tw), fw));
  }
}

// ft_tools.hpp:180-217 (downsample_complex; polar grids via :228-236)
template <bool POLAR>
__global__ void k_ft_downsample(const float* __restrict__ s0, const float* __restrict__ s1, float* __restrict__ d0,
                                float* __restrict__ d1, int T, int F, int dt, int df, int DT, int DF, int preserve) {
  const long long total = (long long)DT * DF;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / DF), f = (int)(i - (long long)t * DF);
    const int tb = t * dt, te = min(tb + dt, T), fb = f * df, fe = min(fb + df, F);
    float2 acc = make_float2(0.f, 0.f);
    int count = 0;
    for (int a = tb; a < te; ++a)
      for (int b = fb; b < fe; ++b) {
        const float2 v = load_c<POLAR>(s0, s1, (long long)a * F + b);
        acc = make_float2(__fadd_rn(acc.x, v.x), __fadd_rn(acc.y, v.y));
        ++count;
      }
    if (preserve && count > 0) {
      const float inv = 1.0f / (float)count;
      acc = make_float2(__fmul_rn(acc.x, inv), __fmul_rn(acc.y, inv));
    }
    store_c<POLAR>(d0, d1, i, acc);
  }
}

// ExponentialHarmonicQuantizer (ft_tools.hpp:257-351)
__device__ __forceinline__ float quant_weight(const QuantP& q, float freq) {
  if (q.mix <= 0.f) return 0.f;
  if (q.base_frequency <= 0.f) return fminf(fmaxf(q.mix, 0.f), 1.f);
  const float ratio = freq / q.base_frequency;
  if (!isfinite((double)ratio)) return 0.f;
  const float nearest = (float)round((double)ratio);
  const float distance = fabsf(__fsub_rn(ratio, nearest));
  const float attraction = expf(__fmul_rn(-q.distance_decay, distance));
  return fminf(fmaxf(__fmul_rn(q.mix, attraction), 0.f), 1.f);
}
__device__ __forceinline__ float quant_magnitude(const QuantP& q, float m, float freq) {
  const float w = quant_weight(q, freq);
  if (w <= 0.f) return m;
  float target = m;
  if (q.magnitude_step > 0.f) target = __fmul_rn((float)round((double)(m / q.magnitude_step)), q.magnitude_step);
  return lerp_rn(m, target, w);
}

template <bool POLAR>
__global__ void k_ft_quantize(float* __restrict__ a0, float* __restrict__ a1, int T, int F, double freq_origin,
                              double freq_step, QuantP q) {
  const long long total = (long long)T * F;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i % F);
    const float freq = (float)(freq_origin + freq_step * (double)f);
    if (POLAR) {
      a0[i] = quant_magnitude(q, a0[i], freq);
    } else {
      const float2 v = make_float2(a0[i], a1[i]);
      const float m = cabs_c(v);
      if (m <= FLT_EPSILON) continue;
      const float adj = quant_magnitude(q, m, freq);
      const float2 o = polar_c(fmaxf(adj, 0.f), carg_c(v));
      a0[i] = o.x;
      a1[i] = o.y;
    }
  }
}

// SpectralLocalContrastBooster (ft_tools.hpp:352-461)
__global__ void k_ft_magnitude(const float* __restrict__ re, const float* __restrict__ im, float* __restrict__ mag,
                               long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    mag[i] = cabs_c(make_float2(__ldg(re + i), __ldg(im + i)));
}

// FP64 sums over whole axes: colsum[f] = sum_t mag[t][f] (thread per column),
// rowsum[t] = sum_f mag[t][f] (block per row, fixed reduction order)
__global__ void k_ft_colsum(const float* __restrict__ mag, double* __restrict__ colsum, int T, int F) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < F; f += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int t = 0; t < T; ++t) s += (double)__ldg(mag + (long long)t * F + f);
    colsum[f] = s;
  }
}
__global__ void __launch_bounds__(256) k_ft_rowsum(const float* __restrict__ mag, double* __restrict__ rowsum, int T,
                                                   int F) {
  __shared__ double part[256];
  for (int t = blockIdx.x; t < T; t += gridDim.x) {
    double s = 0.0;
    for (int f = threadIdx.x; f < F; f += 256) s += (double)__ldg(mag + (long long)t * F + f);
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) rowsum[t] = part[0];
    __syncthreads();
  }
}
// total = sum_t rowsum[t], one block, fixed order
__global__ void __launch_bounds__(256) k_ft_total(const double* __restrict__ rowsum, double* __restrict__ total,
                                                  int T) {
  __shared__ double part[256];
  double s = 0.0;
  for (int t = threadIdx.x; t < T; t += 256) s += rowsum[t];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = part[0];
}

// mode 0: window sums cell by cell (time outer, freq inner, float, as the
// reference); 1: whole grid (mean of the FP64 total); 2: whole time axis x
// freq window (FP64 column sums); 3: time window x whole freq axis (FP64 row
// sums).
__global__ void k_ft_contrast(const float* __restrict__ mag, float* __restrict__ out, int T, int F, int rt, int rf,
                              int mode, const double* __restrict__ sums, ContrastP p) {
  const long long total = (long long)T * F;
  const float gamma_safe = p.gamma > 0.f ? p.gamma : 1.f;
  const bool use_gamma = fabsf(__fsub_rn(gamma_safe, 1.f)) > 1e-5f;
  const float inv_gamma = use_gamma ? 1.f / gamma_safe : 1.f;
  const float gmean = (mode == 1) ? __fdiv_rn((float)sums[0], (float)total) : 0.f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i / F), f = (int)(i - (long long)t * F);
    float mean;
    if (mode == 1) {
      mean = gmean;
    } else if (mode == 0) {
      const int t0 = max(0, t - rt), t1 = min(T - 1, t + rt), f0 = max(0, f - rf), f1 = min(F - 1, f + rf);
      float s = 0.f;
      for (int a = t0; a <= t1; ++a)
        for (int b = f0; b <= f1; ++b) s = __fadd_rn(s, __ldg(mag + (long long)a * F + b));
      mean = __fdiv_rn(s, (float)((t1 - t0 + 1) * (f1 - f0 + 1)));
    } else if (mode == 2) {
      const int f0 = max(0, f - rf), f1 = min(F - 1, f + rf);
      double s = 0.0;
      for (int b = f0; b <= f1; ++b) s += sums[b];
      mean = __fdiv_rn((float)s, (float)((long long)T * (f1 - f0 + 1)));
    } else {
      const int t0 = max(0, t - rt), t1 = min(T - 1, t + rt);
      double s = 0.0;
      for (int a = t0; a <= t1; ++a) s += sums[a];
      mean = __fdiv_rn((float)s, (float)((long long)F * (t1 - t0 + 1)));
    }
    const float cur = __ldg(mag + i);
    const float centered = __fsub_rn(cur, mean);
    const float boosted = __fadd_rn(mean, __fmul_rn(centered, __fadd_rn(1.f, p.contrast)));
    float adj = __fadd_rn(boosted, p.brightness);
    if (p.clamp_zero) adj = fmaxf(adj, 0.f);
    if (use_gamma) adj = (float)pow((double)fmaxf(adj, 1e-12f), (double)inv_gamma);
    out[i] = adj;
  }
}

// complex grid after the booster: polar(new magnitude, arg of the old value)
__global__ void k_ft_repolar(float* __restrict__ re, float* __restrict__ im, const float* __restrict__ mag,
                             long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 o = polar_c(__ldg(mag + i), carg_c(make_float2(re[i], im[i])));
    re[i] = o.x;
    im[i] = o.y;
  }
}

unsigned grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)std::max<long long>(b, 1);
}

void ok(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error("cuda");
}

// per-device working set of the grid pipeline
struct GridWork {
  std::mutex mu;
  cudaStream_t stream = nullptr;
  DevBuf a0, a1, b0, b1, mag, mag2, sums;
};

GridWork& work_for_device() {
  static std::mutex m;
  static std::map<int, GridWork*> all;
  int dev = 0;
  ok(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(m);
  GridWork*& w = all[dev];
  if (!w) {
    w = new GridWork();
    ok(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
  }
  return *w;
}

template <bool POLAR>
int run_pipeline(const ft_grid_spec* spec, const ft_resample_plan_c* plan, const ft_quantizer_config* quant,
                 const ft_contrast_config* contrast, float* u0, float* u1, int T, int F) {
  // ft_tools_cffi.cpp:19-74: defaults of the spec and the plan, shape check
  if (!u0 || !u1 || T <= 0 || F <= 0 || (long long)T * (long long)F >= 0x7fffffffLL) return 0;
  double freq_origin = 0.0, freq_step = 1.0;
  if (spec) {
    freq_origin = spec->freq_origin;
    freq_step = spec->freq_step != 0.0 ? spec->freq_step : 1.0;
  }
  int ut = 1, uf = 1, dt = 1, df = 1, preserve = 1;
  if (plan) {
    ut = plan->upsample_time > 0 ? plan->upsample_time : 1;
    uf = plan->upsample_freq > 0 ? plan->upsample_freq : 1;
    dt = plan->downsample_time > 0 ? plan->downsample_time : 1;
    df = plan->downsample_freq > 0 ? plan->downsample_freq : 1;
    preserve = plan->preserve_energy != 0;
  }
  const bool up = ut > 1 || uf > 1, down = dt > 1 || df > 1;
  const long long UT = up ? (long long)T * ut : T, UF = up ? (long long)F * uf : F;
  const long long DT = down ? (UT + dt - 1) / dt : UT, DF = down ? (UF + df - 1) / df : UF;
  // The reference runs the units and then rejects a grid of another shape,
  // leaving the arrays as they were; nothing observable differs from
  // rejecting it first.
  if (DT != T || DF != F) return 0;
  if (UT * UF >= 0x7fffffffLL) return 0;
  try {
    GridWork& w = work_for_device();
    std::lock_guard<std::mutex> lk(w.mu);
    cudaStream_t s = w.stream;
    const size_t n = (size_t)T * F, un = (size_t)(UT * UF);
    float* c0 = static_cast<float*>(w.a0.get(un * sizeof(float)));
    float* c1 = static_cast<float*>(w.a1.get(un * sizeof(float)));
    ok(cudaMemcpyAsync(c0, u0, n * sizeof(float), cudaMemcpyDefault, s));
    ok(cudaMemcpyAsync(c1, u1, n * sizeof(float), cudaMemcpyDefault, s));
    int ct = T, cf = F;
    if (up) {
      float* n0 = static_cast<float*>(w.b0.get(un * sizeof(float)));
      float* n1 = static_cast<float*>(w.b1.get(un * sizeof(float)));
      k_ft_upsample<POLAR><<<grid_for((long long)un), 256, 0, s>>>(c0, c1, n0, n1, T, F, ut, uf);
      ok(cudaGetLastError());
      // the upsampled grid becomes the current one (a*), b* free again
      std::swap(w.a0.p, w.b0.p);
      std::swap(w.a0.cap, w.b0.cap);
      std::swap(w.a1.p, w.b1.p);
      std::swap(w.a1.cap, w.b1.cap);
      c0 = n0;
      c1 = n1;
      ct = (int)UT;
      cf = (int)UF;
      freq_step /= (double)uf;
    }
    const long long cn = (long long)ct * cf;
    if (quant && quant->enabled && quant->mix > 0.f) {
      const QuantP q{quant->base_frequency, quant->magnitude_step, quant->mix, quant->distance_decay};
      k_ft_quantize<POLAR><<<grid_for(cn), 256, 0, s>>>(c0, c1, ct, cf, freq_origin, freq_step, q);
      ok(cudaGetLastError());
    }
    if (contrast && contrast->enabled) {
      const bool gt = contrast->kernel_time <= 0, gf = contrast->kernel_freq <= 0;
      const int rt = gt ? ct : std::max(contrast->kernel_time / 2, 0);
      const int rf = gf ? cf : std::max(contrast->kernel_freq / 2, 0);
      float* mag = c0;
      if (!POLAR) {
        mag = static_cast<float*>(w.mag.get((size_t)cn * sizeof(float)));
        k_ft_magnitude<<<grid_for(cn), 256, 0, s>>>(c0, c1, mag, cn);
        ok(cudaGetLastError());
      }
      int mode = 0;
      double* sums = nullptr;
      if (gt && gf) {
        mode = 1;
        sums = static_cast<double*>(w.sums.get(((size_t)ct + 1) * sizeof(double)));
        k_ft_rowsum<<<(unsigned)std::min(ct, 148 * 16), 256, 0, s>>>(mag, sums + 1, ct, cf);
        k_ft_total<<<1, 256, 0, s>>>(sums + 1, sums, ct);
      } else if (gt) {
        mode = 2;
        sums = static_cast<double*>(w.sums.get((size_t)cf * sizeof(double)));
        k_ft_colsum<<<grid_for(cf), 256, 0, s>>>(mag, sums, ct, cf);
      } else if (gf) {
        mode = 3;
        sums = static_cast<double*>(w.sums.get((size_t)ct * sizeof(double)));
        k_ft_rowsum<<<(unsigned)std::min(ct, 148 * 16), 256, 0, s>>>(mag, sums, ct, cf);
      }
      ok(cudaGetLastError());
      const ContrastP p{contrast->brightness, contrast->contrast, contrast->gamma, contrast->clamp_zero != 0};
      float* out = static_cast<float*>(w.mag2.get((size_t)cn * sizeof(float)));
      k_ft_contrast<<<grid_for(cn), 256, 0, s>>>(mag, out, ct, cf, rt, rf, mode, sums, p);
      ok(cudaGetLastError());
      if (POLAR) {
        ok(cudaMemcpyAsync(c0, out, (size_t)cn * sizeof(float), cudaMemcpyDeviceToDevice, s));
      } else {
        k_ft_repolar<<<grid_for(cn), 256, 0, s>>>(c0, c1, out, cn);
        ok(cudaGetLastError());
      }
    }
    if (down) {
      float* n0 = static_cast<float*>(w.b0.get(n * sizeof(float)));
      float* n1 = static_cast<float*>(w.b1.get(n * sizeof(float)));
      k_ft_downsample<POLAR><<<grid_for((long long)n), 256, 0, s>>>(c0, c1, n0, n1, ct, cf, dt, df, T, F, preserve);
      ok(cudaGetLastError());
      c0 = n0;
      c1 = n1;
    }
    ok(cudaMemcpyAsync(u0, c0, n * sizeof(float), cudaMemcpyDefault, s));
    ok(cudaMemcpyAsync(u1, c1, n * sizeof(float), cudaMemcpyDefault, s));
    ok(cudaStreamSynchronize(s));
    return 1;
  } catch (...) {
    return 0;
  }
}

}  // namespace
}  // namespace ffb

extern "C" {

FFT_CFFI_API int ft_apply_complex_pipeline(const ft_grid_spec* spec, const ft_resample_plan_c* plan,
                                           const ft_quantizer_config* quant, const ft_contrast_config* contrast,
                                           float* real, float* imag, int time_bins, int freq_bins) {
  return ffb::run_pipeline<false>(spec, plan, quant, contrast, real, imag, time_bins, freq_bins);
}

FFT_CFFI_API int ft_apply_polar_pipeline(const ft_grid_spec* spec, const ft_resample_plan_c* plan,
                                         const ft_quantizer_config* quant, const ft_contrast_config* contrast,
                                         float* magnitude, float* phase, int time_bins, int freq_bins) {
  return ffb::run_pipeline<true>(spec, plan, quant, contrast, magnitude, phase, time_bins, freq_bins);
}

}  // extern "C"
