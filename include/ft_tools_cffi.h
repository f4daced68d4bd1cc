/* ft_tools_cffi.h -- the spectrogram-grid pipeline of the reference's
 * ft_tools C API (ft_tools_cffi.hpp:9-59: same structs, same field order,
 * same entry points), exported by the drop-in libfft_cffi.so and run on the
 * GPU: bilinear upsampling, the exponential harmonic quantizer, the local
 * contrast booster and box downsampling of a time x freq grid (row-major,
 * time_bins rows of freq_bins values), complex (planar re / im) or polar
 * (magnitude / phase).  The arrays are host or device pointers; results
 * replace them in place.  Returns 1 on success, 0 on invalid arguments or
 * when the resampling plan does not return the grid to its own shape (the
 * arrays are then left untouched, as in the reference). */
#pragma once

#include "fft_cffi.h"

#ifdef __cplusplus
extern "C" {
#endif

struct ft_grid_spec {
  double time_origin;
  double freq_origin;
  double time_step; /* 0 -> 1 */
  double freq_step; /* 0 -> 1 */
};

struct ft_resample_plan_c {
  int upsample_time; /* <= 0 -> 1 */
  int upsample_freq;
  int downsample_time;
  int downsample_freq;
  int preserve_energy;
};

struct ft_quantizer_config {
  int enabled;
  float base_frequency;
  float magnitude_step;
  float mix;
  float distance_decay;
};

struct ft_contrast_config {
  int enabled;
  int kernel_time; /* <= 0: the whole time axis */
  int kernel_freq; /* <= 0: the whole freq axis */
  float brightness;
  float contrast;
  float gamma;
  int clamp_zero;
};

/* ft_tools_cffi.cpp:76-124 */
FFT_CFFI_API int ft_apply_complex_pipeline(const struct ft_grid_spec* spec, const struct ft_resample_plan_c* plan,
                                           const struct ft_quantizer_config* quant,
                                           const struct ft_contrast_config* contrast, float* real, float* imag,
                                           int time_bins, int freq_bins);

/* ft_tools_cffi.cpp:126-174 */
FFT_CFFI_API int ft_apply_polar_pipeline(const struct ft_grid_spec* spec, const struct ft_resample_plan_c* plan,
                                         const struct ft_quantizer_config* quant,
                                         const struct ft_contrast_config* contrast, float* magnitude, float* phase,
                                         int time_bins, int freq_bins);

#ifdef __cplusplus
}
#endif
