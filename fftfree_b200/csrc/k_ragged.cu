// k_ragged.cu -- one persistent launch over a ragged batch of real
// transforms (R2C, half spectrum) of different sizes.
//
// Each item i is a signal of N_i = 2^L samples transformed as one full
// frame (window = hop = N_i), exactly as fft_execute_batched does for a
// context of that size (fft_cffi.cpp:701-824); outputs are the planar
// (re, im, mag) rows of N_i/2 + 1 bins, concatenated in item order.
//
// The host builds a work list of tiles, largest first (longest processing
// time first balances the persistent blocks): a tile is either a group of
// same-size items of up to 2^12 complex points, one per S::T-thread slice
// of the 256-thread block (the single-pass engine and the STFT load/store
// policy, so these items match fft_execute_batched bit for bit), or one
// item of 2^13 .. 2^15 complex points, which the block transforms in three
// phases through its own global scratch (columns, rows, untangle; one slot
// of 2^15 points per block, rewritten in place).  Blocks
// take tiles from an atomic counter until the list is exhausted.
#include "fft_launch.cuh"

namespace ffb {
namespace {

constexpr int kBlock = 256;
constexpr int kLargeMin = 13, kLargeMax = 15;  // log2 complex points of the three-phase path

template <class S>
__host__ __device__ constexpr int rtile() {
  return ((S::SMEM + 15) / 16) * 16 + 1;  // 1 mod 16: lanes on different tiles, different banks
}

// ---------------------------------------------------------------- single-pass tile
template <class S, int MODE>
__device__ __forceinline__ void ragged_single(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
  constexpr int T = S::T;
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  const bool ok = g < tile.y;
  const int item = tile.x + (ok ? g : 0);
  const long long po = __ldg(a.pcm_off + item), oo = __ldg(a.out_off + item);
  StftArgs sa{};
  sa.pcm = a.pcm + po;
  sa.pcm_len = 2LL * S::M;
  sa.frames = ok ? 1 : 0;
  sa.N = 2 * S::M;
  sa.W = sa.N;
  sa.H = sa.N;
  sa.pf = a.pf;
  sa.out_bins = S::M + 1;
  sa.out_stride = S::M + 1;
  sa.mag_from_real = 1;
  sa.out_re = a.out_re + oo;
  sa.out_im = a.out_im + oo;
  sa.out_mag = a.out_mag + oo;
  const StftIO<MODE> io{sa, S::LOGM + 1};
  float2* sm = smem + g * S::SMEM;
  float2 v[S::R];
  io.template load<S>(0, t, v, sm, tw);
  fft_engine<S, GroupSync>(v, t, sm, tw);
  io.template store<S>(0, t, v, sm, tw);
}

// ---------------------------------------------------------------- three-phase tile
// z[m] = (x[2m], x[2m+1]), M = M1 * M2 points, m = n1 M2 + n2, k = k1 + M1 k2.
template <int LM1, int LM2, int MODE>
__device__ __forceinline__ void ragged_large(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
  constexpr int LM = LM1 + LM2, M = 1 << LM, M1 = 1 << LM1, M2 = 1 << LM2;
  using SA = Sched<LM1, LM1 - 4>;  // 16 threads per column
  using SB = Sched<LM2, LM2 - 4>;  // 16 threads per row
  static_assert(SA::T == 16 && SB::T == 16, "16 threads per sub-transform");
  const int item = tile.x;
  const float* x = a.pcm + __ldg(a.pcm_off + item);
  const long long oo = __ldg(a.out_off + item);
  // one slot of M points per block: phase A writes the columns' results in
  // row order, phase B overwrites each group of 16 rows, in place, with their
  // results in [k2][row] order (contiguous stores), phase C reads Z[k] at
  // zidx(k).  (A slot per block of M points keeps all blocks' scratch,
  // 444 x 256 KiB, inside the 126 MB L2.)
  float2* scr_a = a.scratch + (long long)blockIdx.x * (1LL << kLargeMax);
  const auto zidx = [](int k) -> long long {
    const int k1 = k & (M1 - 1), k2 = k >> LM1;
    return (long long)(k1 >> 4) * 16 * M2 + (long long)k2 * 16 + (k1 & 15);
  };
  float2* tiles = smem;
  float2* stage = smem + 16 * rtile<SA>();
  // phase A: 16 columns at a time, 16 threads each (lanes walk n2)
  {
    const bool x8 = (reinterpret_cast<uintptr_t>(x) & 7) == 0;
    const int c = threadIdx.x & 15, t = threadIdx.x >> 4;
#pragma unroll 1
    for (int c0 = 0; c0 < M2; c0 += 16) {
      const int n2 = c0 + c;
      float2 v[SA::R];
      if (x8) {  // z[m] = (x[2m], x[2m+1]) as one 8-byte load
        const float2* x2 = reinterpret_cast<const float2*>(x);
#pragma unroll
        for (int i = 0; i < SA::R; ++i) v[i] = __ldg(x2 + (long long)(t + 16 * i) * M2 + n2);
      } else {
#pragma unroll
        for (int i = 0; i < SA::R; ++i) {
          const long long m = (long long)(t + 16 * i) * M2 + n2;
          v[i] = make_float2(__ldg(x + 2 * m), __ldg(x + 2 * m + 1));
        }
      }
      fft_engine<SA, BlockSync>(v, t, tiles + c * rtile<SA>(), tw);
#pragma unroll
      for (int i = 0; i < SA::R; ++i) {
        const int k1 = t + 16 * i;
        scr_a[(long long)k1 * M2 + n2] = cmul(v[i], tw_split(tw, LM, (unsigned)(n2 * k1)));
      }
    }
  }
  __syncthreads();
  // phase B: 16 rows at a time, 16 consecutive lanes per row (lanes walk n2);
  // results staged so that the writes of Z[k1 + M1 k2] walk k1
  {
    const int j = threadIdx.x >> 4, t = threadIdx.x & 15;
#pragma unroll 1
    for (int r0 = 0; r0 < M1; r0 += 16) {
      const int k1 = r0 + j;
      float2 v[SB::R];
#pragma unroll
      for (int i = 0; i < SB::R; ++i) v[i] = scr_a[(long long)k1 * M2 + t + 16 * i];
      fft_engine<SB, BlockSync>(v, t, tiles + j * rtile<SB>(), tw);
#pragma unroll
      for (int i = 0; i < SB::R; ++i) stage[(t + 16 * i) * 17 + j] = v[i];
      __syncthreads();
      // rows r0 .. r0+15 are in registers: their region takes the results
      for (int flat = threadIdx.x; flat < 16 * M2; flat += kBlock) {
        const int k2 = flat >> 4, jj = flat & 15;
        scr_a[(long long)r0 * M2 + flat] = stage[k2 * 17 + jj];
      }
      __syncthreads();
    }
  }
  // phase C: untangle X[k] = E + w_N^k O from Z[k], Z[M - k]; post hook and
  // planar stores as fft_execute_batched's epilogue (fft_cffi.cpp:813-824)
  StftArgs sa{};
  sa.N = 2 * M;
  sa.pf = a.pf;
  sa.mag_from_real = 1;
  const StftIO<MODE> io{sa, LM + 1};
  const bool mag_is_re = (MODE == 1) || (MODE == 2);
  float* re = a.out_re + oo;
  float* im = a.out_im + oo;
  float* mg = a.out_mag + oo;
  const float2* w = tw.pyr + ((2u << LM) - 1u);  // level log2 N
  for (int k = threadIdx.x; k <= M; k += kBlock) {
    if (k == M) {
      const float2 z0 = scr_a[zidx(0)];
      io.emit(re, im, mg, M, make_float2(z0.x - z0.y, 0.f), true, 1.0f, mag_is_re);
      continue;
    }
    const float2 zk = scr_a[zidx(k)];
    const float2 zm = scr_a[zidx((M - k) & (M - 1))];
    const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 D = make_float2(zk.x - zm.x, zk.y + zm.y);
    const float2 O = make_float2(0.5f * D.y, -0.5f * D.x);
    const float2 X = cadd(E, cmul(__ldg(w + k), O));
    io.emit(re, im, mg, k, X, k == 0, 1.0f, mag_is_re);
  }
  __syncthreads();  // scratch and tiles are reused by the block's next tile
}

// ---------------------------------------------------------------- dispatch
// tile.z = log2 complex points, tile.w = pass radix (log2) of a single-pass tile.
template <int MODE>
__device__ __forceinline__ void ragged_tile(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
#define FFB_RS(L, R)                                              \
  case (L) * 8 + (R):                                            \
    ragged_single<Sched<L, R>, MODE>(a, tile, smem, tw);         \
    return;
  switch (tile.z * 8 + tile.w) {
    FFB_RS(1, 2) FFB_RS(2, 2) FFB_RS(3, 2) FFB_RS(4, 2)
    FFB_RS(5, 2) FFB_RS(5, 3) FFB_RS(6, 3) FFB_RS(6, 4) FFB_RS(7, 3) FFB_RS(7, 4)
    FFB_RS(8, 3) FFB_RS(8, 4) FFB_RS(9, 3) FFB_RS(9, 4) FFB_RS(10, 3) FFB_RS(10, 4)
    FFB_RS(11, 3) FFB_RS(11, 4) FFB_RS(12, 4)
    case 13 * 8: ragged_large<7, 6, MODE>(a, tile, smem, tw); return;
    case 14 * 8: ragged_large<7, 7, MODE>(a, tile, smem, tw); return;
    case 15 * 8: ragged_large<8, 7, MODE>(a, tile, smem, tw); return;
    default: return;
  }
#undef FFB_RS
}

template <int MODE>
__global__ void __launch_bounds__(kBlock, 3) k_ragged(RaggedArgs a, Twiddles tw) {
  extern __shared__ float2 smem[];
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int id = next;
    __syncthreads();  // every thread has read `next` before thread 0 overwrites it
    if (id >= a.ntiles) break;
    ragged_tile<MODE>(a, __ldg(a.tiles + id), smem, tw);
  }
}

constexpr size_t ragged_smem_bytes() {
  // single-pass: one 256-thread tile of at most 2^12 points; three-phase:
  // 16 column / row tiles of up to 256 points plus the 128 x 17 staging
  constexpr size_t single = (size_t)4608 * sizeof(float2);  // max over sizes of (256 / T) * S::SMEM
  constexpr size_t large = (size_t)(16 * rtile<Sched<8, 4>>() + 128 * 17) * sizeof(float2);
  return single > large ? single : large;
}

template <int MODE>
cudaError_t launch_mode(const RaggedArgs& a, int grid, cudaStream_t st, uint64_t* launches) {
  const size_t smem = ragged_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_ragged<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  Twiddles tw{twiddle_pyramid(kLargeMax + 1, st), twiddle_pass_tables(st)};
  k_ragged<MODE><<<grid, kBlock, smem, st>>>(a, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

}  // namespace

int ragged_max_log() { return kLargeMax + 1; }  // log2 N of the largest item
bool ragged_large_log(int logm) { return logm >= kLargeMin && logm <= kLargeMax; }
size_t ragged_scratch_per_block() { return (1ull << kLargeMax) * sizeof(float2); }

int ragged_candidates(int logm, int* lrs) {
  if (logm >= kLargeMin) return 0;
  if (logm <= 4) { lrs[0] = 2; return 1; }
  if (logm == 5) { lrs[0] = 2; lrs[1] = 3; return 2; }
  if (logm == 12) { lrs[0] = 4; return 1; }
  lrs[0] = 3;
  lrs[1] = 4;
  return 2;
}

int ragged_grid() {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(k_ragged<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ragged_smem_bytes());
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_ragged<1>, kBlock, ragged_smem_bytes()) != cudaSuccess ||
      per <= 0) {
    cudaGetLastError();
    per = 1;
  }
  return sms * per;
}

cudaError_t launch_ragged(const RaggedArgs& a, int grid, cudaStream_t st, uint64_t* launches) {
  switch (post_mode(a.pf)) {
    case 2: return launch_mode<2>(a, grid, st, launches);
    case 1: return launch_mode<1>(a, grid, st, launches);
    default: return launch_mode<0>(a, grid, st, launches);
  }
}

}  // namespace ffb
