// k_tc05.cu -- batched 256-point complex DFTs on the fifth-generation tensor
// cores: tcgen05.mma (kind::f16, one CTA) with the accumulators in tensor
// memory, in split FP16.  A precision variant of the C2C path at N = 256,
// selected by FFTFREE_TC16=2 (off by default: measured against the FP32
// engine, whose results it must match within the parity bar).
//
// 256 = 16 x 16: with n = 16 n1 + n2 and k = k1 + 16 k2,
//   Y[k1][n2] = sum_n1 w16^(n1 k1) x[16 n1 + n2]           (stage 1)
//   Y[k1][n2] *= w256^(n2 k1)                              (twiddle, FP32)
//   X[k1 + 16 k2] = sum_n2 w16^(n2 k2) Y[k1][n2]           (stage 2)
// Each stage is one real GEMM D[128 x 32] = A[128 x 32] B[32 x 32]^T over a
// tile of 8 transforms: row j of a transform's 16 rows of A holds the 16
// complex inputs of one 16-point DFT as 32 reals (re, im interleaved) --
// x[16 n1 + j] over n1 in stage 1, Y[j][n2] over n2 in stage 2 -- and B is
// the real form of the 16-point DFT matrix (row 2k + c: component c of bin
// k).  With P = P_hi + P_lo split into FP16, D = A_hi B_hi + A_hi B_lo +
// A_lo B_hi (the A_lo B_lo term, about 2^-22 relative, is dropped),
// accumulated in FP32 in tensor memory by six MMAs (three products, two
// K = 16 steps) that one thread issues; a tcgen05.commit arrives on an
// mbarrier that the block waits on (bounded).  Before each split a
// transform's values are scaled by a power of two that puts the largest
// component in [0.5, 1): FP16's range is never exceeded and the split keeps
// 22 bits relative to the transform's maximum.
//
// Operands live in shared memory in the no-swizzle K-major layout of the MMA
// descriptors: 8-row x 16-byte core matrices, the two of one K = 16 step
// 128 B apart (leading byte offset), consecutive 8-row groups 512 B apart
// (stride byte offset).  Single-GPU code: no cluster; every copy is one CTA's own.
#include <cuda_fp16.h>

#include <cstdlib>

#include "kernels.h"
#include "tc16.cuh"

namespace ffb {
namespace {

constexpr int kTcThreads = 128;           // four warps: tensor-memory lanes 0..127
constexpr int kTcTile = 8;                // transforms per tile: 8 x 16 rows = M 128
constexpr unsigned kTcWaitLimit = 1u << 22;  // mbarrier polls before a block gives up

__device__ unsigned g_tc05_timeouts;

// Byte offset of element (m, k) of a 32-column K-major FP16 operand.
__device__ __forceinline__ int op_byte(int m, int k) {
  return (m >> 3) * 512 + (k >> 3) * 128 + (m & 7) * 16 + (k & 7) * 2;
}

struct __align__(128) TcSmem {
  uint4 a_hi[128 * 32 * 2 / 16];  // 8 KB each
  uint4 a_lo[128 * 32 * 2 / 16];
  uint4 b_hi[32 * 32 * 2 / 16];  // 2 KB each
  uint4 b_lo[32 * 32 * 2 / 16];
  unsigned long long bar;
  uint32_t tmem;
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100 format): start address, leading
// byte offset 128, stride byte offset 512 (each >> 4), version 1, no
// swizzle.  K step s starts 256 B further on (two core matrices).
__device__ __forceinline__ uint64_t op_desc(const void* base, int s) {
  const uint32_t a = saddr(base) + 256u * (uint32_t)s;
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(512u >> 4) << 32) |
         (1ull << 46);
}

// Instruction descriptor: D F32 (bits 4-5 = 1), A and B F16 (0), both
// K-major, N = 32 (bits 17-22 = N / 8), M = 128 (bits 24-28 = M / 16).
constexpr uint32_t kIdesc = (1u << 4) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
      : "memory");
}

// D = A_hi B_hi + A_hi B_lo + A_lo B_hi, then a commit to the barrier.
__device__ __forceinline__ void issue_stage(const TcSmem& sm, uint32_t d, uint32_t bar) {
  const void* as[3] = {sm.a_hi, sm.a_hi, sm.a_lo};
  const void* bs[3] = {sm.b_hi, sm.b_lo, sm.b_hi};
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int s = 0; s < 2; ++s) umma(d, op_desc(as[p], s), op_desc(bs[p], s), (p | s) ? 1u : 0u);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, unsigned limit) {
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Row (lanes of this warp) x 32 columns of FP32 accumulators.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&d)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) d[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// The power-of-two exponent e with max(|v|) * 2^-e in [0.5, 1) over the 16
// lanes of one transform (0 for an all-zero transform), clamped so that the
// scale stays a normal float.
__device__ __forceinline__ int group_exponent(float mx) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  int e = 0;
  if (mx > 0.f) frexpf(mx, &e);
  return e < -100 ? -100 : (e > 100 ? 100 : e);
}

__global__ void __launch_bounds__(kTcThreads)
    k_fft256_tc05(const float2* __restrict__ in, float2* __restrict__ out, long long batch, int inverse,
                  Twiddles tw) {
  __shared__ TcSmem sm;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t bar = saddr(&sm.bar);
  // B: the real form of the 16-point DFT matrix, split, one (re, im) input
  // pair (columns 2 n1, 2 n1 + 1) of one output row per step
  for (int e = tid; e < 32 * 16; e += kTcThreads) {
    const int row = e >> 4, n1 = e & 15;
    const int k1 = row >> 1, c = row & 1;
    const float2 w = tw_get(tw, 4, (unsigned)(k1 * n1));  // (Fr, Fi)
    // output re: xr Fr - xi Fi; output im: xr Fi + xi Fr
    const float v0 = c ? w.y : w.x, v1 = c ? w.x : -w.y;
    uint32_t hi, lo;
    split2(v0, v1, &hi, &lo);
    const int off = op_byte(row, 2 * n1);
    *reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(sm.b_hi) + off) = hi;
    *reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(sm.b_lo) + off) = lo;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(saddr(&sm.tmem))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = sm.tmem;
  const uint32_t lanes = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 rows
  const int b = tid >> 4, j = tid & 15;
  const float sg = inverse ? -1.f : 1.f;
  uint32_t phase = 0;
  bool ok = true;
  const long long tiles = (batch + kTcTile - 1) / kTcTile;
  char* ahi = reinterpret_cast<char*>(sm.a_hi);
  char* alo = reinterpret_cast<char*>(sm.a_lo);
  // row tid of a tile's stage 1 operand: x[16 n1 + j], n1 = 0..15
  // (conjugated for the inverse, which is conj . forward . conj / N); the
  // next tile's are fetched while this tile's second stage runs
  float2 x[16];
  const auto fetch = [&](long long t) {
    const long long r = t * kTcTile + b;
    const bool lv = t < tiles && r < batch;
    const float2* src = in + (lv ? r : 0) * 256 + j;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) x[n1] = lv ? __ldg(src + 16 * n1) : make_float2(0.f, 0.f);
  };
  fetch(blockIdx.x);
  for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const long long tr = tile * kTcTile + b;
    const bool live = tr < batch;
    float mx = 0.f;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
      x[n1].y *= sg;
      mx = fmaxf(mx, fmaxf(fabsf(x[n1].x), fabsf(x[n1].y)));
    }
    const int e1 = group_exponent(mx);
    const float s1 = ldexpf(1.f, -e1);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t h[4], l[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) split2(x[4 * q + i].x * s1, x[4 * q + i].y * s1, &h[i], &l[i]);
      const int off = op_byte(tid, 8 * q);
      *reinterpret_cast<uint4*>(ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) issue_stage(sm, tmem, bar);
    ok = __syncthreads_and(bar_wait(bar, phase, kTcWaitLimit));
    phase ^= 1u;
    if (!ok) break;
    fence_after();
    float d[32];
    tmem_ld32(lanes, d);  // Y[k1][j], k1 = 0..15, of transform b (scaled by s1)
    // ---- twiddles w256^(j k1) in FP32, then the stage 2 operand: row
    // (b, k1) = Y[k1][n2] over n2, so this thread writes column j of 16 rows
    float2 y[16];
    float my = 0.f;
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
      const float2 w = tw_get(tw, 8, (unsigned)(j * k1));
      y[k1] = cmul(make_float2(d[2 * k1], d[2 * k1 + 1]), w);
      my = fmaxf(my, fmaxf(fabsf(y[k1].x), fabsf(y[k1].y)));
    }
    fetch(tile + gridDim.x);
    const int e2 = group_exponent(my);
    const float s2 = ldexpf(1.f, -e2);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
      uint32_t h, l;
      split2(y[k1].x * s2, y[k1].y * s2, &h, &l);
      const int off = op_byte(b * 16 + k1, 2 * j);
      *reinterpret_cast<uint32_t*>(ahi + off) = h;
      *reinterpret_cast<uint32_t*>(alo + off) = l;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    if (tid == 0) issue_stage(sm, tmem, bar);
    ok = __syncthreads_and(bar_wait(bar, phase, kTcWaitLimit));
    phase ^= 1u;
    if (!ok) break;
    fence_after();
    tmem_ld32(lanes, d);  // Z[j][k2], k2 = 0..15: bin j + 16 k2 (scaled by s1 s2)
    if (live) {
      const float un = ldexpf(inverse ? 1.f / 256.f : 1.f, e1 + e2);
      float2* dst = out + tr * 256 + j;
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) dst[16 * k2] = make_float2(d[2 * k2] * un, sg * d[2 * k2 + 1] * un);
    }
    // the next tile's operand writes and MMAs come after every thread's
    // reads of this tile's accumulators
    fence_before();
    __syncthreads();
    fence_after();
  }
  if (!ok) {
    // gave up on an MMA commit: count it (the host fails the call), then wait
    // (bounded, 16x longer) for the MMAs still in flight before the tensor
    // memory is released
    if (tid == 0) {
      atomicAdd(&g_tc05_timeouts, 1u);
      (void)bar_wait(bar, phase ^ 1u, 16u * kTcWaitLimit);
    }
    fence_before();
    __syncthreads();
    fence_after();
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}

}  // namespace

bool tc05_requested() {
  const char* e = std::getenv("FFTFREE_TC16");
  return e && e[0] == '2';
}

cudaError_t launch_c2c256_tc05(const C2cArgs& a, cudaStream_t s, uint64_t* launches) {
  if (a.N != 256 || a.pre != 0) return cudaErrorInvalidValue;
  if (a.batch <= 0) return cudaSuccess;
  const long long tiles = (a.batch + kTcTile - 1) / kTcTile;
  const long long grid = tiles < 148 * 4 ? tiles : 148 * 4;
  Twiddles tw{twiddle_pyramid(0, s), twiddle_pass_tables(s)};
  k_fft256_tc05<<<(unsigned)grid, kTcThreads, 0, s>>>(a.in, a.out, a.batch, a.inverse, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

unsigned tc05_timeouts() {
  unsigned v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc05_timeouts, sizeof(v)) != cudaSuccess) return ~0u;
  return v;
}

}  // namespace ffb
