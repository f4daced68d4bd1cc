// fft_engine.cuh -- register/shared-memory FFT engine for sm_100a.
//
// One transform of M = 2^LOGM complex points is held by a group of
// T = M / R threads, R points per thread in registers.  The transform runs
// as a sequence of radix-R Stockham (self-sorting) passes -- preceded by one
// smaller-radix pass when LOGM is not a multiple of log2 R -- with the data
// exchanged between passes through the group's shared-memory tile.  The
// pass arithmetic follows the published Stockham formulation for GPUs
// (Govindaraju et al., SC08):
//   pass with sub-size Ns:  j = thread, k = j mod Ns,
//   v[r] = in[j + r*M/R] * w_{Ns*R}^{k*r};  v = DFT_R(v);
//   out[(j/Ns)*Ns*R + k + r*Ns] = v[r].
// Input layout: v[i] = x[t + i*T];  output layout: v[i] = X[t + i*T]
// (natural order, no final exchange).
//
// This replaces the reference's radix-2 executors (eigen_fft.hpp:2655-3100
// Cooley-Tukey, :3227-3623 Stockham): the transform computed is the same DFT
// (forward sign -1), the stage structure is radix 4/8/16.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ffb {

// ---------------------------------------------------------------- complex
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// -i * a
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }

// ---------------------------------------------------------------- twiddles
// Twiddle pyramid in global memory: level L (0 <= L <= TW_MAX_LOG) holds
// w_L[e] = exp(-2*pi*i*e / 2^L), e < 2^L, at offset 2^L - 1.  Built on the
// host in FP64 with octant symmetry (exact 0 / +-1 at the quarter points).
struct Twiddles {
  const float2* __restrict__ base;
};

__device__ __forceinline__ float2 tw_get(const Twiddles& tw, int L, unsigned e) {
  return __ldg(tw.base + ((1u << L) - 1u) + (e & ((1u << L) - 1u)));
}

// 16th roots of unity (cos, sin of 2*pi*m/16), m = 0..15.
__device__ __forceinline__ float2 w16(int m) {
  // exp(-2*pi*i*m/16) = (cos, -sin)
  constexpr float c1 = 0.92387953251128675613f;  // cos(pi/8)
  constexpr float s1 = 0.38268343236508977173f;  // sin(pi/8)
  constexpr float h = 0.70710678118654752440f;   // sqrt(1/2)
  switch (m & 15) {
    case 0: return make_float2(1.f, 0.f);
    case 1: return make_float2(c1, -s1);
    case 2: return make_float2(h, -h);
    case 3: return make_float2(s1, -c1);
    case 4: return make_float2(0.f, -1.f);
    case 5: return make_float2(-s1, -c1);
    case 6: return make_float2(-h, -h);
    case 7: return make_float2(-c1, -s1);
    case 8: return make_float2(-1.f, 0.f);
    case 9: return make_float2(-c1, s1);
    case 10: return make_float2(-h, h);
    case 11: return make_float2(-s1, c1);
    case 12: return make_float2(0.f, 1.f);
    case 13: return make_float2(s1, c1);
    case 14: return make_float2(h, h);
    default: return make_float2(c1, s1);
  }
}

// ---------------------------------------------------------------- small DFTs
// Forward DFT of R points held in v[stride*0 .. stride*(R-1)], in place,
// natural order in and out.
template <int R, int S = 1>
struct Dft;

template <int S>
struct Dft<1, S> {
  __device__ __forceinline__ static void run(float2*) {}
};

template <int S>
struct Dft<2, S> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a = v[0];
    v[0] = cadd(a, v[S]);
    v[S] = csub(a, v[S]);
  }
};

template <int S>
struct Dft<4, S> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a0 = cadd(v[0], v[2 * S]);
    const float2 a1 = csub(v[0], v[2 * S]);
    const float2 a2 = cadd(v[S], v[3 * S]);
    const float2 a3 = mul_mi(csub(v[S], v[3 * S]));
    v[0] = cadd(a0, a2);
    v[2 * S] = csub(a0, a2);
    v[S] = cadd(a1, a3);
    v[3 * S] = csub(a1, a3);
  }
};

template <int S>
struct Dft<8, S> {
  __device__ __forceinline__ static void run(float2* v) {
    // 2 x 4: DFT4 over even and odd points, then radix-2 combine.
    float2 e[4] = {v[0], v[2 * S], v[4 * S], v[6 * S]};
    float2 o[4] = {v[S], v[3 * S], v[5 * S], v[7 * S]};
    Dft<4, 1>::run(e);
    Dft<4, 1>::run(o);
    constexpr float h = 0.70710678118654752440f;
    const float2 o1 = make_float2((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h);
    const float2 o2 = mul_mi(o[2]);
    const float2 o3 = make_float2((o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h);
    v[0] = cadd(e[0], o[0]);
    v[4 * S] = csub(e[0], o[0]);
    v[S] = cadd(e[1], o1);
    v[5 * S] = csub(e[1], o1);
    v[2 * S] = cadd(e[2], o2);
    v[6 * S] = csub(e[2], o2);
    v[3 * S] = cadd(e[3], o3);
    v[7 * S] = csub(e[3], o3);
  }
};

template <int S>
struct Dft<16, S> {
  __device__ __forceinline__ static void run(float2* v) {
    // 4 x 4: X[k1 + 4 k2] = sum_n2 w4^(n2 k2) w16^(n2 k1) sum_n1 x[4 n1 + n2] w4^(n1 k1)
    float2 a[16];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      a[4 * n2 + 0] = v[(n2)*S];
      a[4 * n2 + 1] = v[(4 + n2) * S];
      a[4 * n2 + 2] = v[(8 + n2) * S];
      a[4 * n2 + 3] = v[(12 + n2) * S];
      Dft<4, 1>::run(a + 4 * n2);
    }
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2) {
#pragma unroll
      for (int k1 = 1; k1 < 4; ++k1) {
        const int m = n2 * k1;
        if (m == 4) a[4 * n2 + k1] = mul_mi(a[4 * n2 + k1]);
        else a[4 * n2 + k1] = cmul(a[4 * n2 + k1], w16(m));
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 b[4] = {a[k1], a[4 + k1], a[8 + k1], a[12 + k1]};
      Dft<4, 1>::run(b);
      v[(k1)*S] = b[0];
      v[(k1 + 4) * S] = b[1];
      v[(k1 + 8) * S] = b[2];
      v[(k1 + 12) * S] = b[3];
    }
  }
};

// ---------------------------------------------------------------- schedule
template <int LOGM_, int LOGR_>
struct Sched {
  static constexpr int LOGM = LOGM_;
  static constexpr int M = 1 << LOGM;
  static constexpr int LOGR = (LOGR_ < LOGM) ? LOGR_ : LOGM;
  static constexpr int R = 1 << LOGR;
  static constexpr int T = M / R;                        // threads per transform
  static constexpr int NFULL = (LOGR > 0) ? LOGM / LOGR : 0;  // full radix-R passes
  static constexpr int LOGR0 = (LOGR > 0) ? LOGM % LOGR : 0;  // leading small pass
};

// XOR swizzle of a shared-memory float2 index: flips the low 4 bits with the
// next 4.  A bijection on every aligned block of 16, it makes the strided
// Stockham write patterns and the unit-stride reads bank-conflict free.
__device__ __forceinline__ int sw(int a) { return a ^ ((a >> 4) & 15); }

// The engine.  `sm` is this group's tile of M float2; `bar` synchronises all
// groups of the block (every thread of the block calls the engine).
template <class S>
__device__ __forceinline__ void fft_engine(float2 (&v)[S::R], int t, float2* sm, const Twiddles& tw) {
  constexpr int M = S::M, R = S::R, T = S::T;
  int Ns = 1;
  int logNs = 0;
  if constexpr (S::LOGR0 > 0) {
    constexpr int r0 = 1 << S::LOGR0;
    constexpr int Q = R / r0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      float2 u[r0];
#pragma unroll
      for (int r = 0; r < r0; ++r) u[r] = v[q + r * Q];
      Dft<r0, 1>::run(u);
      const int j = t + q * T;
#pragma unroll
      for (int r = 0; r < r0; ++r) sm[sw(j * r0 + r)] = u[r];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = sm[sw(t + i * T)];
    __syncthreads();
    Ns = r0;
    logNs = S::LOGR0;
  }
#pragma unroll
  for (int p = 0; p < S::NFULL; ++p) {
    const int k = t & (Ns - 1);
    if (p > 0 || S::LOGR0 > 0) {
      const int L = logNs + S::LOGR;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw_get(tw, L, (unsigned)(k * r)));
    }
    Dft<R, 1>::run(v);
    if (p == S::NFULL - 1) break;
    const int base = ((t >> logNs) << (logNs + S::LOGR)) + k;
#pragma unroll
    for (int r = 0; r < R; ++r) sm[sw(base + r * Ns)] = v[r];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = sm[sw(t + i * T)];
    __syncthreads();
    Ns <<= S::LOGR;
    logNs += S::LOGR;
  }
  (void)M;
}

}  // namespace ffb
