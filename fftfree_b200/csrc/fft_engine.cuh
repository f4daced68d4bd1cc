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
// sm_100a specifics: complex additions use the packed FP32x2 instructions
// (__fadd2_rn / __ffma2_rn, one instruction per complex add); the shared
// tile is padded by one float2 per 16 (conflict-free for every pass
// pattern) so that each element's offset from a per-thread base is a
// compile-time constant; per-pass twiddles come from r-major tables
// (coalesced loads with immediate offsets).
//
// This replaces the reference's radix-2 executors (eigen_fft.hpp:2655-3100
// Cooley-Tukey, :3227-3623 Stockham): the transform computed is the same DFT
// (forward sign -1), the stage structure is radix 4/8/16.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

namespace ffb {

// ---------------------------------------------------------------- complex
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);  // a - b, one rounding
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * b rounded term by term (no contraction into FMA): the same bits in
// every kernel that inlines it, also when b is a compile-time constant
__device__ __forceinline__ float2 cmul_rn(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// -i * a
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }

// ---------------------------------------------------------------- twiddles
// Two FP64-built tables in global memory (host side: kernels.cu):
//  * pyramid: level L (0 <= L <= 18) holds w_L[e] = exp(-2*pi*i*e / 2^L),
//    e < 2^L, at offset 2^L - 1 (untangle and four-step twiddles);
//  * pass tables: for radix R = 2^lr and sub-size Ns = 2^lns the R-1 rows
//    w[(r-1)*Ns + k] = exp(-2*pi*i*k*r / (Ns*R)), k < Ns.
constexpr int kPassMaxLog = 12;  // largest log2(Ns) of a single-pass kernel

__host__ __device__ constexpr long long pass_table_offset(int lr, int lns) {
  long long off = 0;
  for (int l = 1; l < lr; ++l) off += (long long)((1 << l) - 1) * ((1LL << (kPassMaxLog + 1)) - 1);
  return off + (long long)((1 << lr) - 1) * ((1LL << lns) - 1);
}
constexpr long long pass_table_size() { return pass_table_offset(6, 0); }  // radices 2..32

struct Twiddles {
  const float2* __restrict__ pyr;
  const float2* __restrict__ pass;
};

__device__ __forceinline__ float2 tw_get(const Twiddles& tw, int L, unsigned e) {
  return __ldg(tw.pyr + ((1u << L) - 1u) + (e & ((1u << L) - 1u)));
}

// exp(-2 pi i e / 2^L) for the inter-pass twiddles of the multi-pass
// kernels, as the product of two short runs of the pyramid:
// w_{2^L}^e = w_{2^(L-LH)}^(e >> LH) * w_{2^L}^(e & (2^LH - 1)), LH = ceil(L/2).
// A warp's exponents n2 * k1 scatter over the whole level-L table; the two
// factors come from 2^(L-LH) and 2^LH contiguous entries that stay in L1
// (one extra rounding: the product of two correctly rounded factors).
__device__ __forceinline__ float2 tw_split(const Twiddles& tw, int L, unsigned e) {
  const int LH = (L + 1) >> 1;
  const unsigned mask = (1u << L) - 1u;
  e &= mask;
  const float2 hi = __ldg(tw.pyr + ((1u << (L - LH)) - 1u) + (e >> LH));
  const float2 lo = __ldg(tw.pyr + ((1u << L) - 1u) + (e & ((1u << LH) - 1u)));
  return cmul(hi, lo);
}

// exp(-2*pi*i*m/16)
__device__ __forceinline__ float2 w16(int m) {
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

// exp(-2*pi*i*m/32), 0 <= m < 16
__device__ __forceinline__ float2 w32(int m) {
  constexpr float c1 = 0.98078528040323044913f;  // cos(pi/16)
  constexpr float s1 = 0.19509032201612826785f;  // sin(pi/16)
  constexpr float c3 = 0.83146961230254523708f;  // cos(3pi/16)
  constexpr float s3 = 0.55557023301960222474f;  // sin(3pi/16)
  switch (m) {
    case 1: return make_float2(c1, -s1);
    case 3: return make_float2(c3, -s3);
    case 5: return make_float2(s3, -c3);
    case 7: return make_float2(s1, -c1);
    case 9: return make_float2(-s1, -c1);
    case 11: return make_float2(-s3, -c3);
    case 13: return make_float2(-c3, -s3);
    case 15: return make_float2(-c1, -s1);
    default: return w16(m >> 1);
  }
}

// exp(-2*pi*i*m/64) for odd m < 32
__device__ __forceinline__ float2 w64_odd(int m) {
  constexpr float c1 = 0.99518472667219688624f;  // cos(pi/32)
  constexpr float s1 = 0.09801714032956060199f;  // sin(pi/32)
  constexpr float c3 = 0.95694033573220886494f;  // cos(3pi/32)
  constexpr float s3 = 0.29028467725446236764f;  // sin(3pi/32)
  constexpr float c5 = 0.88192126434835502971f;  // cos(5pi/32)
  constexpr float s5 = 0.47139673682599764856f;  // sin(5pi/32)
  constexpr float c7 = 0.77301045336273696081f;  // cos(7pi/32)
  constexpr float s7 = 0.63439328416364549822f;  // sin(7pi/32)
  switch (m) {
    case 1: return make_float2(c1, -s1);
    case 3: return make_float2(c3, -s3);
    case 5: return make_float2(c5, -s5);
    case 7: return make_float2(c7, -s7);
    case 9: return make_float2(s7, -c7);
    case 11: return make_float2(s5, -c5);
    case 13: return make_float2(s3, -c3);
    case 15: return make_float2(s1, -c1);
    case 17: return make_float2(-s1, -c1);
    case 19: return make_float2(-s3, -c3);
    case 21: return make_float2(-s5, -c5);
    case 23: return make_float2(-s7, -c7);
    case 25: return make_float2(-c7, -s7);
    case 27: return make_float2(-c5, -s5);
    case 29: return make_float2(-c3, -s3);
    default: return make_float2(-c1, -s1);  // 31
  }
}

// exp(-2*pi*i*m/64) for any m (a compile-time m folds to a constant)
__device__ __forceinline__ float2 w64(int m) {
  m &= 63;
  const float sg = (m >= 32) ? -1.f : 1.f;  // w^(m + 32) = -w^m
  m &= 31;
  const float2 r = ((m & 1) == 0) ? w32(m >> 1) : w64_odd(m);
  return make_float2(sg * r.x + 0.f, sg * r.y + 0.f);  // + 0: no negative zeros
}

// exp(-2 pi i m / L) for L = 2..64
template <int L>
__device__ __forceinline__ float2 wconst(int m) {
  static_assert(L >= 1 && L <= 64 && (L & (L - 1)) == 0, "L a power of two up to 64");
  return w64(m * (64 / L));
}

// Untangle / Hermitian twiddle w_N^(t + i T) of a transform of M = N/2
// points held as v[i] = point t + i T: w_N^t (one load per thread) times
// w_{2R}^i (a compile-time constant, since N / T = 2R), rounded term by term.
template <class S>
struct UntangleTw {
  float2 wt;
  __device__ __forceinline__ UntangleTw(const Twiddles& tw, int t)
      : wt(__ldg(tw.pyr + ((2u << S::LOGM) - 1u) + t)) {}
  __device__ __forceinline__ float2 operator()(int i) const {
    return i == 0 ? wt : cmul_rn(wt, wconst<2 * S::R>(i));
  }
  // w_N^(t + i T) / 2, the factor of the fused untangles: the halving is
  // folded into the constant (exact), the product taken as two FMAs with
  // explicit roundings (the same bits in every kernel that inlines it).
  __device__ __forceinline__ float2 half(int i) const {
    if (i == 0) return make_float2(0.5f * wt.x, 0.5f * wt.y);
    const float2 c = wconst<2 * S::R>(i);
    const float2 h = make_float2(0.5f * c.x, 0.5f * c.y);
    return make_float2(__fmaf_rn(wt.x, h.x, -__fmul_rn(wt.y, h.y)), __fmaf_rn(wt.x, h.y, __fmul_rn(wt.y, h.x)));
  }
};

// Real-input untangle of one bin: with Z the M-point transform of
// z[m] = x[2m] + i x[2m+1], zk = Z[k], zm = Z[M-k] and h = w_N^k / 2,
//   X[k] = (zk + conj zm) / 2 + h (-i) (zk - conj zm)
// in five FMA-class instructions (explicit roundings, no contraction left
// to the compiler).
__device__ __forceinline__ float2 untangle_bin(float2 zk, float2 zm, float2 h) {
  const float2 A = __ffma2_rn(zm, make_float2(1.f, -1.f), zk);   // zk + conj zm
  const float2 B = __ffma2_rn(zm, make_float2(-1.f, 1.f), zk);   // zk - conj zm
  // h * (-i B) = h * (B.y, -B.x)
  const float2 P = make_float2(__fmaf_rn(h.x, B.y, __fmul_rn(h.y, B.x)), __fmaf_rn(h.y, B.y, -__fmul_rn(h.x, B.x)));
  return __ffma2_rn(A, make_float2(0.5f, 0.5f), P);
}

// ---------------------------------------------------------------- small DFTs
// Forward DFT of R points held in v[0 .. R-1], in place, natural order.
template <int R>
struct Dft;

template <>
struct Dft<1> {
  __device__ __forceinline__ static void run(float2*) {}
};

template <>
struct Dft<2> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a = v[0];
    v[0] = cadd(a, v[1]);
    v[1] = csub(a, v[1]);
  }
};

template <>
struct Dft<4> {
  __device__ __forceinline__ static void run(float2* v) {
    const float2 a0 = cadd(v[0], v[2]);
    const float2 a1 = csub(v[0], v[2]);
    const float2 a2 = cadd(v[1], v[3]);
    const float2 d = csub(v[1], v[3]);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    // a1 -+ i*d
    v[1] = make_float2(a1.x + d.y, a1.y - d.x);
    v[3] = make_float2(a1.x - d.y, a1.y + d.x);
  }
};

template <>
struct Dft<8> {
  __device__ __forceinline__ static void run(float2* v) {
    // 2 x 4: DFT4 over even and odd points, then radix-2 combine.
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4>::run(e);
    Dft<4>::run(o);
    constexpr float h = 0.70710678118654752440f;
    const float2 t1 = make_float2((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h);
    const float2 t3 = make_float2((o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = make_float2(e[2].x + o[2].y, e[2].y - o[2].x);
    v[6] = make_float2(e[2].x - o[2].y, e[2].y + o[2].x);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
  }
};

template <>
struct Dft<16> {
  __device__ __forceinline__ static void run(float2* v) {
    // 4 x 4: X[k1 + 4 k2] = sum_n2 w4^(n2 k2) w16^(n2 k1) sum_n1 x[4 n1 + n2] w4^(n1 k1)
    float2 a[16];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      a[4 * n2 + 0] = v[n2];
      a[4 * n2 + 1] = v[4 + n2];
      a[4 * n2 + 2] = v[8 + n2];
      a[4 * n2 + 3] = v[12 + n2];
      Dft<4>::run(a + 4 * n2);
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
      Dft<4>::run(b);
      v[k1] = b[0];
      v[k1 + 4] = b[1];
      v[k1 + 8] = b[2];
      v[k1 + 12] = b[3];
    }
  }
};

template <>
struct Dft<32> {
  __device__ __forceinline__ static void run(float2* v) {
    // 2 x 16: X[k] = E[k] + w32^k O[k], X[k + 16] = E[k] - w32^k O[k]
    float2 e[16], o[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) {
      e[n] = v[2 * n];
      o[n] = v[2 * n + 1];
    }
    Dft<16>::run(e);
    Dft<16>::run(o);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float2 t = (k == 0) ? o[0] : (k == 8 ? mul_mi(o[8]) : cmul(o[k], w32(k)));
      v[k] = cadd(e[k], t);
      v[k + 16] = csub(e[k], t);
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
  static constexpr int T = M / R;                              // threads per transform
  static constexpr int NFULL = (LOGR > 0) ? LOGM / LOGR : 0;   // full radix-R passes
  static constexpr int LOGR0 = (LOGR > 0) ? LOGM % LOGR : 0;   // leading small pass
  static constexpr int SMEM = M + (M >> 4) + 2;                // padded tile (float2), index M included
};

// Barrier policies of the engine.  BlockSync: the whole block (kernels
// whose blocks share tiles across transforms).  GroupSync: only the S::T
// threads of one transform -- a warp barrier when a transform fits in a
// warp, else a named barrier per group of a block of 256 threads (groups
// are the consecutive S::T-thread slices; at most 4 of them here), or the
// block barrier when one transform is the whole block.
struct BlockSync {
  static constexpr bool kSplitTwiddles = false;  // pass twiddles: full table loads
  template <class S>
  __device__ __forceinline__ static void sync() {
    __syncthreads();
  }
};

// Block barriers for kernels whose transforms are interleaved across the
// lanes of a block, with the twiddle arithmetic of the single-pass kernels
// (bit-identical results to GroupSync engines).
struct LaneBlockSync {
  static constexpr bool kSplitTwiddles = true;
  template <class S>
  __device__ __forceinline__ static void sync() {
    __syncthreads();
  }
};

struct GroupSync {
  static constexpr bool kSplitTwiddles = true;  // rows 1..3 and multiples of 4 loaded, the rest products
  template <class S>
  __device__ __forceinline__ static void sync() {
    if constexpr (S::T <= 32) {
      __syncwarp();
    } else if constexpr (S::T >= 256) {
      __syncthreads();
    } else {
      static_assert(256 / S::T <= 15, "one named barrier per group");
      asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / S::T)), "n"(S::T) : "memory");
    }
  }
};

// Padded shared-memory index: one float2 of padding per 16.
__device__ __forceinline__ int pidx(int a) { return a + (a >> 4); }

// v[i] <- tile[t + i*T]
template <class S>
__device__ __forceinline__ void tile_read(float2 (&v)[S::R], int t, const float2* sm) {
  if constexpr (S::T % 16 == 0) {
    const float2* b = sm + pidx(t);
#pragma unroll
    for (int i = 0; i < S::R; ++i) v[i] = b[i * S::T + ((i * S::T) >> 4)];
  } else {
#pragma unroll
    for (int i = 0; i < S::R; ++i) v[i] = sm[pidx(t + i * S::T)];
  }
}

// tile[t + i*T] <- v[i]
template <class S>
__device__ __forceinline__ void tile_write_natural(const float2 (&v)[S::R], int t, float2* sm) {
  if constexpr (S::T % 16 == 0) {
    float2* b = sm + pidx(t);
#pragma unroll
    for (int i = 0; i < S::R; ++i) b[i * S::T + ((i * S::T) >> 4)] = v[i];
  } else {
#pragma unroll
    for (int i = 0; i < S::R; ++i) sm[pidx(t + i * S::T)] = v[i];
  }
}

template <class S, class Y, int P>
__device__ __forceinline__ void stockham_pass(float2 (&v)[S::R], int t, float2* sm, const Twiddles& tw) {
  constexpr int R = S::R, LR = S::LOGR;
  constexpr int LNS = S::LOGR0 + P * LR;
  constexpr int NS = 1 << LNS;
  const int k = t & (NS - 1);
  if constexpr (LNS > 0 && NS <= 4 && NS * R <= 64) {
    // few distinct twiddles (k < NS): compile-time constants, chosen by k
#pragma unroll
    for (int r = 1; r < R; ++r) {
      float2 w = make_float2(1.f, 0.f);
#pragma unroll
      for (int kk = 1; kk < NS; ++kk)
        if (k == kk) w = wconst<NS * R>(r * kk);
      v[r] = cmul_rn(v[r], w);
    }
  } else if constexpr (LNS > 0 && (R == 8 || R == 16) && Y::kSplitTwiddles) {
    // w^r for r = 4a + b (0 < b < 4) as w^(4a) w^b: the table rows r = 1, 2,
    // 3 and the multiples of 4 are loaded, the rest are one product away.
    // Single-pass kernels only (per-transform barriers): B200 sweeps show it
    // faster there (C2C N=4096 -5%) and slower in the block-synchronised
    // multi-pass kernels (N=65536 +5%).
    const float2* w = tw.pass + pass_table_offset(LR, LNS) + k;
    float2 wb[4], wa[R / 4];
#pragma unroll
    for (int b = 1; b < 4; ++b) wb[b] = __ldg(w + (b - 1) * NS);
#pragma unroll
    for (int a = 1; a < R / 4; ++a) wa[a] = __ldg(w + (4 * a - 1) * NS);
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const int a = r >> 2, b = r & 3;
      const float2 wr = (a == 0) ? wb[b] : (b == 0 ? wa[a] : cmul_rn(wa[a], wb[b]));
      v[r] = cmul(v[r], wr);
    }
  } else if constexpr (LNS > 0) {
    const float2* w = tw.pass + pass_table_offset(LR, LNS) + k;
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(w + (r - 1) * NS));
  }
  Dft<R>::run(v);
  if constexpr (P != S::NFULL - 1) {
    const int base = ((t >> LNS) << (LNS + LR)) + k;
    if constexpr (NS >= 16 || LNS + LR >= 4) {
      // (base + r*NS) >> 4 == (base >> 4) + (r*NS >> 4) for these patterns
      float2* b = sm + pidx(base);
#pragma unroll
      for (int r = 0; r < R; ++r) b[r * NS + ((r * NS) >> 4)] = v[r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) sm[pidx(base + r * NS)] = v[r];
    }
    Y::template sync<S>();
    tile_read<S>(v, t, sm);
    Y::template sync<S>();
  }
}

template <class S, class Y, int... P>
__device__ __forceinline__ void run_passes(float2 (&v)[S::R], int t, float2* sm, const Twiddles& tw,
                                           std::integer_sequence<int, P...>) {
  (stockham_pass<S, Y, P>(v, t, sm, tw), ...);
}

// The engine.  `sm` is this group's padded tile (S::SMEM float2); every
// thread of the block (BlockSync) or of the group (GroupSync) calls it.
template <class S, class Y = BlockSync>
__device__ __forceinline__ void fft_engine(float2 (&v)[S::R], int t, float2* sm, const Twiddles& tw) {
  constexpr int R = S::R, T = S::T;
  if constexpr (S::LOGR0 > 0) {
    constexpr int r0 = 1 << S::LOGR0;
    constexpr int Q = R / r0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      float2 u[r0];
#pragma unroll
      for (int r = 0; r < r0; ++r) u[r] = v[q + r * Q];
      Dft<r0>::run(u);
      const int j = t + q * T;
#pragma unroll
      for (int r = 0; r < r0; ++r) sm[pidx(j * r0 + r)] = u[r];
    }
    Y::template sync<S>();
    tile_read<S>(v, t, sm);
    Y::template sync<S>();
  }
  run_passes<S, Y>(v, t, sm, tw, std::make_integer_sequence<int, S::NFULL>{});
}

}  // namespace ffb
