// k_2d.cu -- the second axis of a 2-D transform (fft_inplace_2d,
// eigen_fft.hpp:3177-3215): C2C lines whose consecutive elements lie `rows`
// complex values apart in a column-major rows x cols matrix.
//
// The reference transposes the matrix into scratch, transforms the now
// contiguous rows and transposes back (three passes over the matrix).  Here
// one kernel does it in a single read and a single write: a block owns G
// adjacent lines (adjacent rows of one matrix) and thread x works on line
// x % G as engine thread x / G, so consecutive threads load and store
// consecutive lines -- adjacent addresses, whole 32-byte sectors for G >= 4
// -- straight between HBM and registers; shared memory only carries the
// engine's exchanges.  When G divides the row count (every block's lines in
// one matrix) the lines move by TMA instead (k_fft_strided_tma: the block's
// whole input in flight at once, measured 1.0-1.25x the load/store form);
// FFTFREE_2D_TMA=0 keeps the load/store form.  Lines longer than the
// single-pass engine (cols > 2^13) take the transpose / multi-pass /
// transpose route.
#include <cuda.h>  // CUtensorMap and the encoder's types (the encoder is reached through the runtime)

#include <cstdlib>

#include "fft_launch.cuh"

namespace ffb {

template <class S, int WANT = 4>
struct LinesLaunch {
  // group stride (float2): the G groups of a half-warp land on disjoint banks
  static constexpr int gstride(int g) {
    const int res = g >= 16 ? 1 : 16 / g;
    return S::SMEM + (((res - S::SMEM % 16) % 16) + 16) % 16;
  }
  static constexpr size_t bytes(int g) { return (size_t)g * gstride(g) * sizeof(float2); }
  static constexpr int pick() {
    int g = (S::T >= 256) ? 1 : 256 / S::T;
    const int want = (1024 / S::T < WANT) ? 1024 / S::T : WANT;  // >= 4 lines: whole sectors
    if (g < want) g = want;
    while (g > 1 && bytes(g) > 200 * 1024) g >>= 1;
    return g;
  }
  static constexpr int G = pick();
  static constexpr int GS = gstride(G);
  static constexpr int BLOCK = S::T * G;
  static constexpr size_t SMEM_BYTES = bytes(G);
};

template <class S, int WANT>
__global__ void __launch_bounds__(LinesLaunch<S, WANT>::BLOCK) k_fft_strided(StridedLinesArgs a, Twiddles tw) {
  using L = LinesLaunch<S, WANT>;
  extern __shared__ float2 smem[];
  constexpr int T = S::T, M = S::M, G = L::G, GS = L::GS;
  static_assert((G & (G - 1)) == 0, "lines per block: a power of two");
  const int g = threadIdx.x & (G - 1);
  const int t = threadIdx.x / G;
  const long long l = (long long)blockIdx.x * G + g;
  const bool live = l < a.c.batch;
  const long long st = a.rows;
  const long long o = live ? (l / st) * st * (long long)M + (l % st) : 0;
  float2 v[S::R];
  // inverse = conj . forward . conj
  const float2 sg_in = make_float2(1.f, a.c.inverse ? -1.f : 1.f);
  if (a.c.pre == 0) {
    const float2* p = a.c.in + o;
#pragma unroll
    for (int i = 0; i < S::R; ++i)
      v[i] = live ? __fmul2_rn(__ldcg(p + (long long)(t + i * T) * st), sg_in) : make_float2(0.f, 0.f);
  } else {
    const float2* p = a.c.in + o;
    const auto at = [p, st](int m) { return __ldcg(p + (long long)m * st); };
#pragma unroll
    for (int i = 0; i < S::R; ++i)
      v[i] = live ? __fmul2_rn(c2c_pre_elem(a.c, at, t + i * T), sg_in) : make_float2(0.f, 0.f);
  }
  // the groups of a block are interleaved across lanes: block barriers
  fft_engine<S, LaneBlockSync>(v, t, smem + g * GS, tw);
  if (!live) return;
  const float sc = a.c.inverse ? 1.0f / (float)M : 1.0f;
  const float2 sg = make_float2(sc, a.c.inverse ? -sc : sc);
  float2* q = a.c.out + o;
  if (!any_post(a.c.pf)) {
#pragma unroll
    for (int i = 0; i < S::R; ++i) __stcg(q + (long long)(t + i * T) * st, __fmul2_rn(v[i], sg));
  } else {
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int k = t + i * T;
      __stcg(q + (long long)k * st, post_hook(__fmul2_rn(v[i], sg), k, M, a.c.pf));
    }
  }
}

// Lines per block wanted (2, 4 or 8; FFTFREE_2D_LINES), before the
// shared-memory cap.  Default from B200 sweeps of the TMA kernel: 2 for
// lines of 4096 points and more (two blocks per SM overlap load, compute
// and store: 3.26 vs 2.89 TB/s at 4096), 4 below (2048: 4.10 vs 3.62).
static int lines_wanted(int logm) {
  static const int env = [] {
    const char* e = std::getenv("FFTFREE_2D_LINES");
    const int v = e ? std::atoi(e) : 0;
    return (v == 2 || v == 4 || v == 8) ? v : 0;
  }();
  if (env) return env;
  return logm >= 12 ? 2 : 4;
}

template <int LOGM, int LOGR, int WANT>
static cudaError_t run_strided_w(const StridedLinesArgs& a, cudaStream_t st, uint64_t* launches) {
  using S = Sched<LOGM, LOGR>;
  if constexpr (S::T > 1024) {
    return cudaErrorInvalidValue;
  } else {
    using L = LinesLaunch<S, WANT>;
    const long long grid = (a.c.batch + L::G - 1) / L::G;
    if (grid <= 0) return cudaSuccess;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
    if (L::SMEM_BYTES > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_fft_strided<S, WANT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)L::SMEM_BYTES);
      if (e != cudaSuccess) return e;
    }
    Twiddles tw{twiddle_pyramid(0, st), twiddle_pass_tables(st)};
    k_fft_strided<S, WANT><<<(unsigned)grid, L::BLOCK, L::SMEM_BYTES, st>>>(a, tw);
    if (launches) ++*launches;
    return cudaGetLastError();
  }
}

// ------------------------------------------------------------------ TMA variant
// The same transform with the G lines moved by the Tensor Memory Accelerator:
// one thread issues boxes of G lines x BN elements (a 3-D tensor map over
// rows x cols x batch, 8-byte elements) into a [n][line] staging tile, the
// whole block's input in flight at once; the result leaves the same way
// through TMA stores.  The engine's tiles reuse the staging space.

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbar_wait_parity(uint32_t bar, uint32_t parity, unsigned limit) {
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

template <class S, int WANT>
__global__ void __launch_bounds__(LinesLaunch<S, WANT>::BLOCK)
    k_fft_strided_tma(const __grid_constant__ CUtensorMap map_in, const __grid_constant__ CUtensorMap map_out,
                      StridedLinesArgs a, Twiddles tw, unsigned first_wait_limit) {
  using L = LinesLaunch<S, WANT>;
  constexpr int G = L::G;
  constexpr int T = S::T, M = S::M, GS = L::GS;
  constexpr int BN = M < 256 ? M : 256;  // elements per box (box: G x BN)
  constexpr unsigned kLimit = 1u << 22;  // try_wait polls before a block gives up
  extern __shared__ __align__(128) float2 smem[];
  float2* stage = smem;  // [M][G] while loading and storing
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + G * GS);
  const uint32_t bar_a = smem_addr(bar);
  const int g = threadIdx.x & (G - 1);
  const int t = threadIdx.x / G;
  const long long l0 = (long long)blockIdx.x * G;
  const int mat = (int)(l0 / a.rows), r0 = (int)(l0 % a.rows);  // G | rows: one matrix
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(G * M * 8) : "memory");
#pragma unroll 1
    for (int n0 = 0; n0 < M; n0 += BN)
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
          "[%5];" ::"r"(smem_addr(stage + n0 * G)),
          "l"(reinterpret_cast<uint64_t>(&map_in)), "r"(r0), "r"(n0), "r"(mat), "r"(bar_a)
          : "memory");
  }
  const bool ok = __syncthreads_and(mbar_wait_parity(bar_a, 0, first_wait_limit));
  if (!ok) {
    // give up: count it for the host (which fails the call), then wait
    // (bounded, 16x longer) for the copies still in flight before the block
    // releases its shared memory; its lines are left unwritten
    if (threadIdx.x == 0) {
      atomicAdd(a.timeouts, 1u);
      (void)mbar_wait_parity(bar_a, 0, 16u * kLimit);
    }
    __syncthreads();
    return;
  }
  float2 v[S::R];
  const float2 sg_in = make_float2(1.f, a.c.inverse ? -1.f : 1.f);  // inverse = conj . forward . conj
  if (a.c.pre == 0) {
#pragma unroll
    for (int i = 0; i < S::R; ++i) v[i] = __fmul2_rn(stage[(t + i * T) * G + g], sg_in);
  } else {
    const auto at = [stage, g](int n) { return stage[n * G + g]; };
#pragma unroll
    for (int i = 0; i < S::R; ++i) v[i] = __fmul2_rn(c2c_pre_elem(a.c, at, t + i * T), sg_in);
  }
  __syncthreads();
  fft_engine<S, LaneBlockSync>(v, t, smem + g * GS, tw);
  __syncthreads();
  const float sc = a.c.inverse ? 1.0f / (float)M : 1.0f;
  const float2 sg = make_float2(sc, a.c.inverse ? -sc : sc);
#pragma unroll
  for (int i = 0; i < S::R; ++i) {
    const int k = t + i * T;
    float2 X = __fmul2_rn(v[i], sg);
    if (any_post(a.c.pf)) X = post_hook(X, k, M, a.c.pf);
    stage[k * G + g] = X;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> async proxy
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll 1
    for (int n0 = 0; n0 < M; n0 += BN)
      asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
                       reinterpret_cast<uint64_t>(&map_out)),
                   "r"(r0), "r"(n0), "r"(mat), "r"(smem_addr(stage + n0 * G))
                   : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // staging tile read out before exit
  }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (EncodeTiledFn) nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// rows x cols x batch matrices of 8-byte elements, box G x bn x 1
static bool make_lines_map(CUtensorMap* m, const void* base, long long rows, long long cols, long long batch, int g,
                           int bn) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)rows, (cuuint64_t)cols, (cuuint64_t)batch};
  const cuuint64_t strides[2] = {(cuuint64_t)rows * 8, (cuuint64_t)(rows * cols) * 8};
  const cuuint32_t box[3] = {(cuuint32_t)g, (cuuint32_t)bn, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Polls of the first input wait before a block gives up.  The full limit
// unless FFTFREE_TEST_TMA_WAIT_LIMIT is set: a test-only override (0 makes
// every block give up at once) that exercises the reporting of a wait that
// ran out; the drain wait keeps its full limit.
static unsigned first_wait_limit() {
  static const unsigned lim = [] {
    const char* e = std::getenv("FFTFREE_TEST_TMA_WAIT_LIMIT");
    return e ? (unsigned)std::strtoul(e, nullptr, 10) : (1u << 22);
  }();
  return lim;
}

static bool tma_wanted() {
  static const bool on = [] {
    const char* e = std::getenv("FFTFREE_2D_TMA");
    return !(e && e[0] == '0');
  }();
  return on;
}

// TMA path when the lines of a block share one matrix (G | rows), the
// strides are 16-byte multiples and both bases 16-byte aligned; returns
// cudaErrorNotSupported to let the caller take the LSU kernel.
template <int LOGM, int LOGR, int WANT>
static cudaError_t run_strided_tma(const StridedLinesArgs& a, cudaStream_t st, uint64_t* launches) {
  using S = Sched<LOGM, LOGR>;
  if constexpr (S::T > 1024) {
    return cudaErrorNotSupported;
  } else {
    using L = LinesLaunch<S, WANT>;
    constexpr int G = L::G;
    constexpr int BN = S::M < 256 ? S::M : 256;
    if (!tma_wanted() || !a.timeouts || G < 2 || a.rows % G != 0 || (reinterpret_cast<uintptr_t>(a.c.in) & 15) ||
        (reinterpret_cast<uintptr_t>(a.c.out) & 15) || a.rows > 0x7fffffffLL)
      return cudaErrorNotSupported;
    const long long batch = a.c.batch / a.rows;
    if (batch * a.rows != a.c.batch || batch > 0x7fffffffLL) return cudaErrorNotSupported;
    CUtensorMap mi, mo;
    if (!make_lines_map(&mi, a.c.in, a.rows, S::M, batch, G, BN) ||
        !make_lines_map(&mo, a.c.out, a.rows, S::M, batch, G, BN))
      return cudaErrorNotSupported;
    const size_t smem = L::SMEM_BYTES + 16;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k_fft_strided_tma<S, WANT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
    }
    const long long grid = a.c.batch / G;
    if (grid > 0x7fffffffLL) return cudaErrorNotSupported;
    Twiddles tw{twiddle_pyramid(0, st), twiddle_pass_tables(st)};
    k_fft_strided_tma<S, WANT><<<(unsigned)grid, L::BLOCK, smem, st>>>(mi, mo, a, tw, first_wait_limit());
    if (launches) ++*launches;
    return cudaGetLastError();
  }
}

template <int LOGM, int LOGR>
static cudaError_t run_strided(const StridedLinesArgs& a, cudaStream_t st, uint64_t* launches) {
  if (a.c.batch > 0) {
    cudaError_t e;
    switch (lines_wanted(LOGM)) {
      case 2: e = run_strided_tma<LOGM, LOGR, 2>(a, st, launches); break;
      case 8: e = run_strided_tma<LOGM, LOGR, 8>(a, st, launches); break;
      default: e = run_strided_tma<LOGM, LOGR, 4>(a, st, launches); break;
    }
    if (e != cudaErrorNotSupported) return e;
  }
  switch (lines_wanted(LOGM)) {
    case 2: return run_strided_w<LOGM, LOGR, 2>(a, st, launches);
    case 8: return run_strided_w<LOGM, LOGR, 8>(a, st, launches);
    default: return run_strided_w<LOGM, LOGR, 4>(a, st, launches);
  }
}

template <int LOGM>
static cudaError_t strided_r(const StridedLinesArgs& a, int logr, cudaStream_t st, uint64_t* l) {
  switch (logr) {
    case 2: return run_strided<LOGM, 2>(a, st, l);
    case 3: return run_strided<LOGM, 3>(a, st, l);
    case 5:
      if constexpr (LOGM >= 9) return run_strided<LOGM, 5>(a, st, l);
      else return run_strided<LOGM, 4>(a, st, l);
    default: return run_strided<LOGM, 4>(a, st, l);
  }
}

int max_strided_log() { return 13; }

cudaError_t launch_c2c_strided(const StridedLinesArgs& a, int req_logr, cudaStream_t s, uint64_t* launches) {
  if (a.rows <= 0) return cudaErrorInvalidValue;
  const int logm = ilog2i(a.c.N);
  const int logr = choose_logr(logm, req_logr, false);
  if (logr < 0) return cudaErrorInvalidValue;
  switch (logm) {
    case 0: return strided_r<0>(a, logr, s, launches);
    case 1: return strided_r<1>(a, logr, s, launches);
    case 2: return strided_r<2>(a, logr, s, launches);
    case 3: return strided_r<3>(a, logr, s, launches);
    case 4: return strided_r<4>(a, logr, s, launches);
    case 5: return strided_r<5>(a, logr, s, launches);
    case 6: return strided_r<6>(a, logr, s, launches);
    case 7: return strided_r<7>(a, logr, s, launches);
    case 8: return strided_r<8>(a, logr, s, launches);
    case 9: return strided_r<9>(a, logr, s, launches);
    case 10: return strided_r<10>(a, logr, s, launches);
    case 11: return strided_r<11>(a, logr, s, launches);
    case 12: return strided_r<12>(a, logr, s, launches);
    case 13: return strided_r<13>(a, logr, s, launches);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------------ transpose
// Column-major rows x cols -> cols x rows for each of `batch` matrices,
// through 32 x 32 shared-memory tiles (coalesced on both sides).
__global__ void __launch_bounds__(256) k_transpose(const float2* __restrict__ in, float2* __restrict__ out,
                                                   long long rows, long long cols, long long batch) {
  __shared__ float2 tile[32][33];
  const long long r0 = (long long)blockIdx.x * 32, c0 = (long long)blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (long long m = blockIdx.z; m < batch; m += gridDim.z) {
    const float2* src = in + m * rows * cols;
    float2* dst = out + m * rows * cols;
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
      const long long r = r0 + tx, c = c0 + ty + j;
      if (r < rows && c < cols) tile[ty + j][tx] = src[r + c * rows];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 32; j += 8) {
      const long long c = c0 + tx, r = r0 + ty + j;
      if (r < rows && c < cols) dst[c + r * cols] = tile[tx][ty + j];
    }
    __syncthreads();
  }
}

cudaError_t launch_transpose(const float2* in, float2* out, long long rows, long long cols, long long batch,
                             cudaStream_t s, uint64_t* launches) {
  if (rows <= 0 || cols <= 0 || batch <= 0) return cudaSuccess;
  const long long gx = (rows + 31) / 32, gy = (cols + 31) / 32;
  if (gx > 0x7fffffffLL || gy > 65535) return cudaErrorInvalidValue;
  const unsigned gz = (unsigned)(batch < 65535 ? batch : 65535);
  k_transpose<<<dim3((unsigned)gx, (unsigned)gy, gz), 256, 0, s>>>(in, out, rows, cols, batch);
  if (launches) ++*launches;
  return cudaGetLastError();
}

}  // namespace ffb
