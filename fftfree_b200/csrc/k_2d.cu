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
// engine's exchanges.  Lines longer than the single-pass engine
// (cols > 2^13) take the transpose / multi-pass / transpose route.
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

// Lines per block wanted (2, 4 or 8; FFTFREE_2D_LINES, default 4), before
// the shared-memory cap.
static int lines_wanted() {
  static const int w = [] {
    const char* e = std::getenv("FFTFREE_2D_LINES");
    const int v = e ? std::atoi(e) : 4;
    return (v == 2 || v == 8) ? v : 4;
  }();
  return w;
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

template <int LOGM, int LOGR>
static cudaError_t run_strided(const StridedLinesArgs& a, cudaStream_t st, uint64_t* launches) {
  switch (lines_wanted()) {
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
