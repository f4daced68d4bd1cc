// The reference's own spectrogram-grid tools (ft_tools.hpp, header only,
// standard C++) built as the checker of the GPU grid pipeline.
//
// TEST INFRASTRUCTURE ONLY: compiled by oracle/Makefile (`make ref`) from the
// header where it lies in the reference tree into oracle/_ref/; never linked
// into the product.  The two entry points restate the glue of
// ft_tools_cffi.cpp:76-174 around the header's units: grid spec and plan
// defaults, the optional units, the shape check and the copies in and out.
#include <complex>
#include <cstddef>
#include <limits>

#include "ft_tools.hpp"

namespace {

using fftfree::ft::ComplexGrid;
using fftfree::ft::PolarGrid;

struct GridSpecC {
  double time_origin, freq_origin, time_step, freq_step;
};
struct PlanC {
  int upsample_time, upsample_freq, downsample_time, downsample_freq, preserve_energy;
};
struct QuantC {
  int enabled;
  float base_frequency, magnitude_step, mix, distance_decay;
};
struct ContrastC {
  int enabled, kernel_time, kernel_freq;
  float brightness, contrast, gamma;
  int clamp_zero;
};

fftfree::ft::GridSpec grid_of(const GridSpecC* g) {
  fftfree::ft::GridSpec s;
  if (!g) return s;
  s.time_origin = g->time_origin;
  s.freq_origin = g->freq_origin;
  s.time_step = g->time_step != 0.0 ? g->time_step : 1.0;
  s.freq_step = g->freq_step != 0.0 ? g->freq_step : 1.0;
  return s;
}

fftfree::ft::ResamplePlan plan_of(const PlanC* p) {
  fftfree::ft::ResamplePlan r;
  if (!p) return r;
  r.upsample_time = p->upsample_time > 0 ? p->upsample_time : 1;
  r.upsample_freq = p->upsample_freq > 0 ? p->upsample_freq : 1;
  r.downsample_time = p->downsample_time > 0 ? p->downsample_time : 1;
  r.downsample_freq = p->downsample_freq > 0 ? p->downsample_freq : 1;
  r.preserve_energy = p->preserve_energy != 0;
  return r;
}

template <class Field>
bool run(const GridSpecC* g, const PlanC* p, const QuantC* q, const ContrastC* c, Field& field, int T, int F) {
  const fftfree::ft::ResamplePlan plan = plan_of(p);
  if (plan.upsample_time > 1 || plan.upsample_freq > 1)
    field = fftfree::ft::upsample_field(field, plan.upsample_time, plan.upsample_freq);
  fftfree::ft::ExponentialHarmonicQuantizer<float> qu;
  fftfree::ft::SpectralLocalContrastBooster<float> co;
  if (q && q->enabled) {
    qu.base_frequency = q->base_frequency;
    qu.magnitude_step = q->magnitude_step;
    qu.mix = q->mix;
    qu.distance_decay = q->distance_decay;
    qu(field);
  }
  if (c && c->enabled) {
    co.kernel_time = c->kernel_time;
    co.kernel_freq = c->kernel_freq;
    co.brightness = c->brightness;
    co.contrast = c->contrast;
    co.gamma = c->gamma;
    co.clamp_zero = c->clamp_zero != 0;
    co(field);
  }
  if (plan.downsample_time > 1 || plan.downsample_freq > 1)
    field = fftfree::ft::downsample_field(field, plan.downsample_time, plan.downsample_freq, plan.preserve_energy);
  return field.time_bins == T && field.freq_bins == F;
}

bool shape_ok(int T, int F) {
  return T > 0 && F > 0 && (long long)T * (long long)F < (long long)std::numeric_limits<int>::max();
}

}  // namespace

extern "C" {

int ref_ft_apply_complex_pipeline(const GridSpecC* g, const PlanC* p, const QuantC* q, const ContrastC* c, float* re,
                                  float* im, int T, int F) {
  if (!re || !im || !shape_ok(T, F)) return 0;
  const std::size_t n = (std::size_t)T * (std::size_t)F;
  ComplexGrid<float> field(T, F, grid_of(g));
  for (std::size_t i = 0; i < n; ++i) field.values[i] = std::complex<float>(re[i], im[i]);
  if (!run(g, p, q, c, field, T, F)) return 0;
  for (std::size_t i = 0; i < n; ++i) {
    re[i] = field.values[i].real();
    im[i] = field.values[i].imag();
  }
  return 1;
}

int ref_ft_apply_polar_pipeline(const GridSpecC* g, const PlanC* p, const QuantC* q, const ContrastC* c, float* mag,
                                float* ph, int T, int F) {
  if (!mag || !ph || !shape_ok(T, F)) return 0;
  const std::size_t n = (std::size_t)T * (std::size_t)F;
  PolarGrid<float> field(T, F, grid_of(g));
  for (std::size_t i = 0; i < n; ++i) {
    field.magnitude[i] = mag[i];
    field.phase[i] = ph[i];
  }
  if (!run(g, p, q, c, field, T, F)) return 0;
  for (std::size_t i = 0; i < n; ++i) {
    mag[i] = field.magnitude[i];
    ph[i] = field.phase[i];
  }
  return 1;
}

}  // extern "C"
