// k_fourstep.cu -- multi-pass (four-step) transforms for sizes beyond one
// thread block: N = N1 * N2 with N1 = 2^ceil(L/2), N2 = 2^floor(L/2),
//   X[k1 + N1 k2] = sum_n2 w_N2^(n2 k2) [ w_N^(n2 k1) sum_n1 x[n1 N2 + n2] w_N1^(n1 k1) ].
// Pass A: column FFTs of length N1 (stride N2) for a tile of C consecutive
//   columns per block (lanes walk consecutive n2, so loads are coalesced),
//   times the inter-pass twiddle w_N^(n2 k1), written row-major (k1, n2)
//   into a scratch chunk.
// Pass B: row FFTs of length N2 for C consecutive rows per block; results are
//   staged through shared memory so that the writes of X[k1 + N1 k2] walk
//   consecutive k1.
// The batch runs in chunks of scratch (chunk * N complex, up to 1 GiB by
// default: one chunk for most batches, both passes then streaming through
// HBM); with several chunks, pass A of the next chunk overlaps pass B of
// the current one on a second stream.
// Each IO policy supplies elem4 (input element n) and emit4 (output bin k)
// with the same hook semantics as the single-pass kernels.
#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "fft_launch.cuh"
#include "tc16.cuh"

namespace ffb {

namespace {

// Shared tile stride per group: padded, and 1 mod 16 so that lanes of
// different groups touching the same in-tile index hit different banks.
template <class S>
__host__ __device__ constexpr int tile_stride() {
  return ((S::SMEM + 15) / 16) * 16 + 1;
}

// Columns per block: the column pass reads C consecutive complex points
// (C * 8 bytes) from each row; FFTFREE_FOURSTEP_COLS (compile time) picks
// the width, bounded by 1024 threads per block.
#ifndef FFTFREE_FOURSTEP_COLS
#define FFTFREE_FOURSTEP_COLS 16
#endif
template <class S>
__host__ __device__ constexpr int cols_for() {
  return (S::T * FFTFREE_FOURSTEP_COLS <= 1024) ? FFTFREE_FOURSTEP_COLS : 1024 / S::T;
}

// The transform of each column / row group: the radix-R engine, or (TC, for
// 256-point groups) the split-FP16 tensor-core DFT of tc16.cuh, one warp per
// group tile.
template <class S, bool TC>
__device__ __forceinline__ void group_fft(float2 (&v)[S::R], int t, float2* smem, int group, int groups,
                                          const Twiddles& tw) {
  float2* tile = smem + group * tile_stride<S>();
  if constexpr (TC && S::LOGM == 8) {
    tile_write_natural<S>(v, t, tile);
    __syncthreads();
    for (int gg = threadIdx.x >> 5; gg < groups; gg += blockDim.x >> 5) tc_fft256(smem + gg * tile_stride<S>(), tw);
    __syncthreads();
    tile_read<S>(v, t, tile);
  } else {
    fft_engine<S>(v, t, tile, tw);
  }
}

template <class S1, class IO, bool TC>
__global__ void __launch_bounds__(S1::T * cols_for<S1>())
k_four_a(IO io, float2* __restrict__ scratch, long long b0, int LN, Twiddles tw) {
  extern __shared__ float2 smem[];
  constexpr int C = cols_for<S1>();
  constexpr int T1 = S1::T;
  constexpr int N1 = S1::M;
  const int N2 = 1 << (LN - S1::LOGM);
  const int c = threadIdx.x % C;
  const int t = threadIdx.x / C;
  const int tiles = N2 / C;
  const long long bl = blockIdx.x / tiles;
  const int n2 = (int)(blockIdx.x % tiles) * C + c;
  const long long b = b0 + bl;
  float2 v[S1::R];
#pragma unroll
  for (int i = 0; i < S1::R; ++i) v[i] = io.elem4(b, (long long)(t + i * T1) * N2 + n2);
  group_fft<S1, TC>(v, t, smem, c, C, tw);
  float2* out = scratch + bl * ((long long)N1 * N2);
#pragma unroll
  for (int i = 0; i < S1::R; ++i) {
    const int k1 = t + i * T1;
    out[(long long)k1 * N2 + n2] = cmul(v[i], tw_split(tw, LN, (unsigned)(n2 * k1)));
  }
}

template <class S2, class IO, bool TC>
__global__ void __launch_bounds__(S2::T * cols_for<S2>())
k_four_b(IO io, const float2* __restrict__ scratch, long long b0, int LN, Twiddles tw) {
  extern __shared__ float2 smem[];
  constexpr int C = cols_for<S2>();
  constexpr int T2 = S2::T;
  constexpr int N2 = S2::M;
  const int N1 = 1 << (LN - S2::LOGM);
  const int g = threadIdx.x / T2;
  const int t = threadIdx.x % T2;
  const int tiles = N1 / C;
  const long long bl = blockIdx.x / tiles;
  const int k1_0 = (int)(blockIdx.x % tiles) * C;
  const float2* row = scratch + bl * ((long long)N1 * N2) + (long long)(k1_0 + g) * N2;
  float2 v[S2::R];
#pragma unroll
  for (int i = 0; i < S2::R; ++i) v[i] = row[t + i * T2];
  group_fft<S2, TC>(v, t, smem, g, C, tw);
  __syncthreads();  // the tiles are reused for staging
#pragma unroll
  for (int i = 0; i < S2::R; ++i) smem[(t + i * T2) * (C + 1) + g] = v[i];
  __syncthreads();
  const long long b = b0 + bl;
  for (int flat = threadIdx.x; flat < C * N2; flat += blockDim.x) {
    const int k2 = flat / C, gg = flat - k2 * C;
    io.emit4(b, (long long)(k1_0 + gg) + (long long)N1 * k2, smem[k2 * (C + 1) + gg]);
  }
}

template <int LN1>
using SubSched = Sched<LN1, 4>;

template <class S>
cudaError_t set_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
}

// Two-stream software pipeline over chunks: pass A of chunk i+1 (stream
// sa) overlaps pass B of chunk i (stream sb); the two scratch slots
// alternate, so A(i) waits for B(i-2).  Forks from and joins back into the
// caller's stream `st` through events.
struct FourStepStreams {
  cudaStream_t sa = nullptr, sb = nullptr;
  cudaEvent_t fork = nullptr, done_a[2] = {nullptr, nullptr}, done_b[2] = {nullptr, nullptr};
  bool ok = false;
};

FourStepStreams& pipeline_streams() {
  // one set per device (the calling thread's current device)
  static std::mutex mu;
  static FourStepStreams per_dev[64];
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  FourStepStreams& p = per_dev[dev & 63];
  if (!p.ok) {
    bool good = cudaStreamCreateWithFlags(&p.sa, cudaStreamNonBlocking) == cudaSuccess &&
                cudaStreamCreateWithFlags(&p.sb, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < 2 && good; ++i)
      good = cudaEventCreateWithFlags(&p.done_a[i], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&p.done_b[i], cudaEventDisableTiming) == cudaSuccess;
    p.ok = good;
  }
  return p;
}

template <int LN1, int LN2, class IO, bool TC = false>
cudaError_t run_four(const IO& io, long long batch, float2* scratch, long long chunk, cudaStream_t st,
                     uint64_t* launches) {
  using S1 = SubSched<LN1>;
  using S2 = SubSched<LN2>;
  constexpr int LN = LN1 + LN2;
  constexpr int C1 = cols_for<S1>(), C2 = cols_for<S2>();
  const size_t sm1 = (size_t)C1 * tile_stride<S1>() * sizeof(float2);
  // pass B also stages its C2 x N2 results with a (C2 + 1) stride
  const size_t sm2 = std::max((size_t)C2 * tile_stride<S2>(), (size_t)S2::M * (C2 + 1)) * sizeof(float2);
  cudaError_t e = set_smem<S1>((const void*)k_four_a<S1, IO, TC>, sm1);
  if (e != cudaSuccess) return e;
  e = set_smem<S2>((const void*)k_four_b<S2, IO, TC>, sm2);
  if (e != cudaSuccess) return e;
  Twiddles tw{twiddle_pyramid(LN, st), twiddle_pass_tables(st)};
  const long long slot = chunk * (1LL << LN);  // complex points per scratch slot
  const long long nchunks = (batch + chunk - 1) / chunk;
  FourStepStreams& p = pipeline_streams();
  static std::mutex enqueue_mu;  // the shared events are re-recorded per call
  std::lock_guard<std::mutex> lk(enqueue_mu);
  const bool pipelined = p.ok && nchunks > 1;
  cudaStream_t sa = pipelined ? p.sa : st, sb = pipelined ? p.sb : st;
  if (pipelined) {
    if ((e = cudaEventRecord(p.fork, st)) != cudaSuccess) return e;
    cudaStreamWaitEvent(sa, p.fork, 0);
    cudaStreamWaitEvent(sb, p.fork, 0);
  }
  for (long long i = 0; i < nchunks; ++i) {
    const long long b0 = i * chunk;
    const long long nb = std::min(chunk, batch - b0);
    const int sl = pipelined ? (int)(i & 1) : 0;
    float2* buf = scratch + sl * slot;
    const long long ga = nb * ((1LL << LN2) / C1);
    const long long gb = nb * ((1LL << LN1) / C2);
    if (pipelined && i >= 2) cudaStreamWaitEvent(sa, p.done_b[sl], 0);
    k_four_a<S1, IO, TC><<<(unsigned)ga, S1::T * C1, sm1, sa>>>(io, buf, b0, LN, tw);
    if (pipelined) {
      cudaEventRecord(p.done_a[sl], sa);
      cudaStreamWaitEvent(sb, p.done_a[sl], 0);
    }
    k_four_b<S2, IO, TC><<<(unsigned)gb, S2::T * C2, sm2, sb>>>(io, buf, b0, LN, tw);
    if (pipelined) cudaEventRecord(p.done_b[sl], sb);
    if (launches) *launches += 2;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (pipelined) {
    // join: the caller's stream continues after both passes of every chunk
    cudaEventRecord(p.fork, sa);
    cudaStreamWaitEvent(st, p.fork, 0);
    cudaEventRecord(p.fork, sb);
    cudaStreamWaitEvent(st, p.fork, 0);
  }
  return cudaGetLastError();
}

template <class IO, bool TC = false>
cudaError_t four_dispatch(const IO& io, int LN, long long batch, float2* scratch, long long chunk,
                          cudaStream_t st, uint64_t* l) {
  switch (LN) {
    case 14: return run_four<7, 7, IO, TC>(io, batch, scratch, chunk, st, l);
    case 15: return run_four<8, 7, IO, TC>(io, batch, scratch, chunk, st, l);
    case 16: return run_four<8, 8, IO, TC>(io, batch, scratch, chunk, st, l);
    case 17: return run_four<9, 8, IO, TC>(io, batch, scratch, chunk, st, l);
    case 18: return run_four<9, 9, IO, TC>(io, batch, scratch, chunk, st, l);
    case 19: return run_four<10, 9, IO, TC>(io, batch, scratch, chunk, st, l);
    case 20: return run_four<10, 10, IO, TC>(io, batch, scratch, chunk, st, l);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

int max_multi_pass_log() { return 20; }

// Scratch is sized for two slots of `chunk` transforms (see run_four).
size_t four_step_chunk(int LN, long long batch) {
  // Scratch budget per chunk (MB; FFTFREE_FOURSTEP_CHUNK_MB overrides it).
  // B200 sweeps: one large chunk beats L2-sized chunks, whose one-wave
  // launches lose more to ramp-up and tail than L2 residency saves.
  static const long long budget_mb = [] {
    const char* e = std::getenv("FFTFREE_FOURSTEP_CHUNK_MB");
    const long long v = e ? std::atoll(e) : 0;
    return v > 0 ? v : 1024LL;
  }();
  const long long per = (1LL << LN) * (long long)sizeof(float2);
  long long chunk = std::max<long long>(1, (budget_mb << 20) / per);
  return (size_t)std::min<long long>(chunk, std::max<long long>(batch, 1));
}

cudaError_t launch_four_step_stft(const StftArgs& a, float2* scratch, size_t chunk, cudaStream_t s,
                                  uint64_t* launches) {
  const int LN = ilog2i(a.N);
  switch (post_mode(a.pf)) {
    case 2: return four_dispatch(StftIO<2>{a, LN}, LN, a.frames, scratch, (long long)chunk, s, launches);
    case 1: return four_dispatch(StftIO<1>{a, LN}, LN, a.frames, scratch, (long long)chunk, s, launches);
    default: return four_dispatch(StftIO<0>{a, LN}, LN, a.frames, scratch, (long long)chunk, s, launches);
  }
}

// FFTFREE_TC16=1 runs the 256-point groups of the C2C multi-pass transforms
// (2^15 .. 2^17 points) on the tensor cores in split FP16 (tc16.cuh); off by
// default: measured slower than the FP32 engine at this accuracy.
bool tc16_requested() {
  const char* e = std::getenv("FFTFREE_TC16");
  return e && e[0] == '1';
}

cudaError_t launch_four_step_c2c(const C2cArgs& a, float2* scratch, size_t chunk, cudaStream_t s,
                                 uint64_t* launches) {
  const int LN = ilog2i(a.N);
  if (tc16_requested() && LN >= 15 && LN <= 17)
    return four_dispatch<C2cIO, true>(C2cIO{a}, LN, a.batch, scratch, (long long)chunk, s, launches);
  return four_dispatch(C2cIO{a}, LN, a.batch, scratch, (long long)chunk, s, launches);
}

cudaError_t launch_four_step_cplx(const CplxBatchArgs& a, float2* scratch, size_t chunk, cudaStream_t s,
                                  uint64_t* launches) {
  return four_dispatch(CplxBatchIO{a}, ilog2i(a.N), a.frames, scratch, (long long)chunk, s, launches);
}

}  // namespace ffb
