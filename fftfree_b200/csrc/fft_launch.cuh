// fft_launch.cuh -- the single-pass batched FFT kernel template and its
// compile-time dispatch over transform size and pass radix.
#pragma once

#include "io.cuh"

namespace ffb {

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
  float2* sm = smem + g * S::SMEM;
  float2 v[S::R];
  io.template load<S>(b, t, v, sm, tw);
  fft_engine<S, GroupSync>(v, t, sm, tw);
  io.template store<S>(b, t, v, sm, tw);
}

template <class S, class IO>
static cudaError_t run(const IO& io, long long nbatch, cudaStream_t st, uint64_t* launches) {
  using L = Launch<S>;
  if (nbatch <= 0) return cudaSuccess;
  const long long grid = (nbatch + L::G - 1) / L::G;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
  const size_t smem = (size_t)L::G * S::SMEM * sizeof(float2);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_fft<S, IO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
  }
  Twiddles tw{twiddle_pyramid(0, st), twiddle_pass_tables(st)};
  k_fft<S, IO><<<(unsigned)grid, L::BLOCK, smem, st>>>(io, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

// Compile-time table of instantiations: LOGM 0..13, LOGR 2..4 (clamped by
// Sched) and 5 from LOGM 9 up, threads per transform <= 1024.
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
    case 5:
      if constexpr (LOGM >= 9) return run_if_valid<IO, LOGM, 5>(io, n, st, l);
      else return run_if_valid<IO, LOGM, 4>(io, n, st, l);
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

inline int ilog2i(long long n) {
  int l = 0;
  while ((1LL << l) < n) ++l;
  return l;
}

}  // namespace ffb
