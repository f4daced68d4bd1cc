// k_ragged.cu -- one persistent launch over a ragged batch of real
// transforms (R2C, half spectrum) of different sizes and framings.
//
// Item i is a signal framed as fft_execute_batched frames it (pad_mode 1,
// fft_cffi.cpp:701-824): frames of W_i samples at hop H_i, zero-padded to
// N_i, windowed by the item's analysis taps; its frames' planar (re, im,
// mag) rows of N_i/2 + 1 bins are concatenated in item order.  Every frame
// is one job; the host groups the jobs of one size into tiles, largest
// first (longest processing time first balances the persistent blocks), and
// the blocks (1024 threads, one per SM) take tiles from an atomic counter
// until the list is exhausted.  A tile is
//  * a group of same-size frames of up to 2^14 complex points, one per
//    T-thread slice of the block, in one or more block-loads taken one after
//    the other (the tile size the tuner picks) -- the single-pass engine and the STFT
//    load / store policy of fft_execute_batched, so a frame matches that
//    call bit for bit where the radix is the same; 2^14 points take the
//    whole block (T = 1024, the transform held in registers and 139 KB of
//    shared memory);
//  * one frame of 2^15 complex points (N = 65536), which exceeds one SM's
//    shared memory: a decimation-in-time split into two 2^14-point
//    transforms of the even and odd points, run one after the other through
//    the block's engine; the first half's spectrum waits in a 128 KB scratch
//    slot of the block (148 slots, 19 MB: L2-resident), and the combine step
//    untangles bins k and k + M/2 together so the outputs stay contiguous.
#include "fft_launch.cuh"

namespace ffb {
namespace {

constexpr int kBlock = 1024;
constexpr int kSplitLog = 15;  // log2 complex points of the two-half path
constexpr int kFullLog = 14;   // one-block single pass

// ---------------------------------------------------------------- single-pass tile
template <class S, int MODE>
__device__ __forceinline__ void ragged_single(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
  constexpr int T = S::T;
  constexpr int G = kBlock / T;  // frames the block holds at once
  static_assert(T <= 32 || kBlock / T <= 15 || T >= 256, "named barrier per group");
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  float2* sm = smem + g * S::SMEM;
  // a tile holds one or more block-loads of frames (the tuner's tile size),
  // taken one after the other by the block's groups
  for (int base = 0; base < tile.y; base += G) {
    if (base > 0) GroupSync::sync<S>();  // the previous frame's store has read the group's tile
    const bool ok = base + g < tile.y;
    const int2 job = __ldg(a.jobs + tile.x + (ok ? base + g : 0));
    const RaggedItem it = a.items[job.x];
    StftArgs sa{};
    sa.pcm = a.pcm + it.pcm_off;
    sa.pcm_len = it.pcm_len;
    sa.frames = ok ? (long long)job.y + 1 : 0;  // frame job.y of the item (none when !ok)
    sa.N = 2 * S::M;
    sa.W = it.W;
    sa.H = it.H;
    sa.win = it.win_off >= 0 ? a.windows + it.win_off : nullptr;
    sa.pf = a.pf;
    sa.out_bins = S::M + 1;
    sa.out_stride = S::M + 1;
    sa.mag_from_real = 1;
    sa.out_re = a.out_re + it.out_off;
    sa.out_im = a.out_im + it.out_off;
    sa.out_mag = a.out_mag + it.out_off;
    const StftIO<MODE> io{sa, S::LOGM + 1};
    float2 v[S::R];
    io.template load<S>(job.y, t, v, sm, tw);
    fft_engine<S, GroupSync>(v, t, sm, tw);
    io.template store<S>(job.y, t, v, sm, tw);
  }
}

// ---------------------------------------------------------------- two-half tile
// Samples j, j + 1 of the windowed, zero-padded frame.
__device__ __forceinline__ float2 frame_pair(const float* src, const float* win, long long cnt, long long j,
                                             bool fast) {
  if (fast) {
    float2 z = __ldg(reinterpret_cast<const float2*>(src + j));
    if (win) z = __fmul2_rn(z, __ldg(reinterpret_cast<const float2*>(win + j)));
    return z;
  }
  float x0 = 0.f, x1 = 0.f;
  if (j < cnt) x0 = win ? __ldg(src + j) * __ldg(win + j) : __ldg(src + j);
  if (j + 1 < cnt) x1 = win ? __ldg(src + j + 1) * __ldg(win + j + 1) : __ldg(src + j + 1);
  return make_float2(x0, x1);
}

// M = 2^15 complex points z[m] = (s[2m], s[2m+1]) of an N = 2^16 frame:
// E = DFT_{M/2}(z[2n]), O = DFT_{M/2}(z[2n+1]),
// Z[k] = E[k] + w_M^k O[k], Z[k + M/2] = E[k] - w_M^k O[k]; then
// X[k] = untangle(Z[k], Z[M - k]) and X[k + M/2] = untangle(Z[k + M/2], Z[M/2 - k]).
// The points z[2n + odd] of the tile's frame into v (n = t + i T).  The
// frame's bookkeeping is re-read for each half, so that nothing but the tile
// stays live across the engine (a 2^14-point engine at 1024 threads uses the
// whole register budget).
template <class S>
__device__ __forceinline__ void split_load(const RaggedArgs& a, int4 tile, int odd, int t, float2 (&v)[S::R]) {
  constexpr int T = S::T, R = S::R, N = 4 * S::M;
  const int2 job = __ldg(a.jobs + tile.x);
  const RaggedItem it = a.items[job.x];
  long long cnt;
  const float* src = stft_frame(a.pcm + it.pcm_off, it.pcm_len, 0, 0, it.W, it.H, job.y, &cnt);
  const float* win = it.win_off >= 0 ? a.windows + it.win_off : nullptr;
  const bool fast = cnt == (long long)N && aligned8(src) && (!win || aligned8(win));
#pragma unroll
  for (int i = 0; i < R; ++i) v[i] = frame_pair(src, win, cnt, 4LL * (t + i * T) + 2 * odd, fast);
}

template <int MODE>
__device__ __forceinline__ void ragged_split(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
  using S = Sched<kSplitLog - 1, 4>;
  constexpr int T = S::T, R = S::R, MH = S::M, M = 2 * MH, LM = kSplitLog;
  static_assert(T == kBlock, "the whole block per half");
  const int t = threadIdx.x;

  // even points: E, into the block's scratch slot; then the odd points: O,
  // into the tile (the engine's barriers also order the scratch writes
  // before the combine's reads).  One engine body for both halves.
#pragma unroll 1
  for (int odd = 0; odd < 2; ++odd) {
    float2 v[R];
    split_load<S>(a, tile, odd, t, v);
    fft_engine<S, GroupSync>(v, t, smem, tw);
    if (odd) {
      tile_write_natural<S>(v, t, smem);
    } else {
      float2* scr = a.scratch + (long long)blockIdx.x * MH;
#pragma unroll
      for (int i = 0; i < R; ++i) scr[t + i * T] = v[i];
    }
  }
  __syncthreads();

  const int2 job = __ldg(a.jobs + tile.x);
  const RaggedItem it = a.items[job.x];
  const float2* scr = a.scratch + (long long)blockIdx.x * MH;

  StftArgs sa{};
  sa.N = 2 * M;
  sa.pf = a.pf;
  sa.mag_from_real = 1;
  const StftIO<MODE> io{sa, LM + 1};
  const bool mag_is_re = (MODE == 1) || (MODE == 2);
  float* re = a.out_re + it.out_off + (long long)job.y * (M + 1);
  float* im = a.out_im + it.out_off + (long long)job.y * (M + 1);
  float* mg = a.out_mag + it.out_off + (long long)job.y * (M + 1);
  // w_M^k and w_N^k for k = t + i T: w^t (one pyramid load per thread) times
  // w_32^i and w_64^i (M / T = 32, N / T = 64), rounded term by term, the
  // latter read from the pyramid's small levels 5 and 6 (the same entry for
  // the whole warp); the large levels (256 and 512 KB) are not read per bin,
  // and the loop stays rolled (the kernel's code already strains the
  // instruction cache)
  static_assert(M / T == 32 && 2 * M / T == 64, "combine twiddles from levels 5 and 6");
  const float2 wMt = tw_get(tw, LM, (unsigned)t);
  const float2 wNt = tw_get(tw, LM + 1, (unsigned)t);
#pragma unroll 2
  for (int i = 0; i < R; ++i) {
    const int k = t + i * T;
    const float2 wk = i == 0 ? wMt : cmul_rn(wMt, tw_get(tw, 5, (unsigned)i));  // w_M^k
    const float2 e = scr[k];
    const float2 o = cmul(smem[pidx(k)], wk);  // O[k] (from the tile: the registers go to the combine)
    const float2 zk = cadd(e, o);                       // Z[k]
    const float2 zk2 = csub(e, o);                      // Z[k + M/2]
    float2 zmk, zmk2;                                   // Z[M - k], Z[M/2 - k]
    if (k == 0) {
      zmk = zk;
      zmk2 = zk2;
    } else {
      const float2 wm = make_float2(-wk.x, wk.y);       // w_M^(M/2 - k) = -conj(w_M^k)
      const float2 om = cmul(smem[pidx(MH - k)], wm);
      const float2 em = scr[MH - k];
      zmk2 = cadd(em, om);
      zmk = csub(em, om);
    }
    const float2 wn = i == 0 ? wNt : cmul_rn(wNt, tw_get(tw, 6, (unsigned)i));  // w_N^k
    const float2 h = make_float2(0.5f * wn.x, 0.5f * wn.y);
    const float2 h2 = make_float2(0.5f * wn.y, -0.5f * wn.x);  // w_N^(k + M/2) / 2 = -i w_N^k / 2
    float2 X = untangle_bin(zk, zmk, h);
    if (k == 0) X.y = 0.f;  // DC
    io.emit(re, im, mg, k, X, k == 0, 1.0f, mag_is_re);
    io.emit(re, im, mg, k + MH, untangle_bin(zk2, zmk2, h2), false, 1.0f, mag_is_re);
    if (k == 0) io.emit(re, im, mg, M, make_float2(zk.x - zk.y, 0.f), true, 1.0f, mag_is_re);  // Nyquist
  }
  __syncthreads();  // shared memory and scratch are reused by the block's next tile
}

// ---------------------------------------------------------------- dispatch
// tile.z = log2 complex points, tile.w = pass radix (log2); the pass radices
// keep T = M / R out of (32, 128) (named barriers per group: 15 at most).
template <int MODE>
__device__ __forceinline__ void ragged_tile(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
#define FFB_RS(L, R)                                              \
  case (L) * 8 + (R):                                            \
    ragged_single<Sched<L, R>, MODE>(a, tile, smem, tw);         \
    return;
  switch (tile.z * 8 + tile.w) {
    FFB_RS(1, 2) FFB_RS(2, 2) FFB_RS(3, 2) FFB_RS(4, 2)
    FFB_RS(5, 2) FFB_RS(5, 3) FFB_RS(6, 3) FFB_RS(6, 4) FFB_RS(7, 3) FFB_RS(7, 4)
    FFB_RS(8, 3) FFB_RS(8, 4) FFB_RS(9, 4) FFB_RS(10, 3)
    FFB_RS(11, 3) FFB_RS(11, 4) FFB_RS(12, 4) FFB_RS(13, 4) FFB_RS(14, 4)
    case kSplitLog * 8: ragged_split<MODE>(a, tile, smem, tw); return;
    default: return;
  }
#undef FFB_RS
}

template <int MODE>
__global__ void __launch_bounds__(kBlock, 1) k_ragged(RaggedArgs a, Twiddles tw) {
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

// Shared memory of a tile of (L, R): one padded tile per T-thread group.
template <int L, int R>
constexpr size_t tile_smem() {
  using S = Sched<L, R>;
  return (size_t)(kBlock / S::T) * S::SMEM * sizeof(float2);
}
constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }

constexpr size_t ragged_smem_bytes() {
  // the largest over the tiles of ragged_tile (small transforms carry more
  // padding per point: 256 groups of 64 points take the most)
  return cmax(cmax(cmax(cmax(tile_smem<1, 2>(), tile_smem<2, 2>()), cmax(tile_smem<3, 2>(), tile_smem<4, 2>())),
                   cmax(cmax(tile_smem<5, 2>(), tile_smem<5, 3>()), cmax(tile_smem<6, 3>(), tile_smem<6, 4>()))),
              cmax(cmax(cmax(tile_smem<7, 3>(), tile_smem<7, 4>()), cmax(tile_smem<8, 3>(), tile_smem<8, 4>())),
                   cmax(cmax(cmax(tile_smem<9, 4>(), tile_smem<10, 3>()), cmax(tile_smem<11, 3>(), tile_smem<11, 4>())),
                        cmax(cmax(tile_smem<12, 4>(), tile_smem<13, 4>()), tile_smem<14, 4>()))));
}
static_assert(ragged_smem_bytes() <= 227 * 1024, "one block per SM");

template <int MODE>
cudaError_t launch_mode(const RaggedArgs& a, int grid, cudaStream_t st, uint64_t* launches) {
  const size_t smem = ragged_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_ragged<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  Twiddles tw{twiddle_pyramid(kSplitLog + 1, st), twiddle_pass_tables(st)};
  k_ragged<MODE><<<grid, kBlock, smem, st>>>(a, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

}  // namespace

int ragged_max_log() { return kSplitLog + 1; }  // log2 N of the largest item
int ragged_block_log(int logm) { return logm >= kFullLog ? 1 : 0; }
size_t ragged_scratch_per_block() { return (size_t)(1u << (kSplitLog - 1)) * sizeof(float2); }
int ragged_block_threads() { return kBlock; }

int ragged_candidates(int logm, int* lrs) {
  if (logm >= kSplitLog) return 0;
  if (logm <= 4) { lrs[0] = 2; return 1; }
  if (logm == 5) { lrs[0] = 2; lrs[1] = 3; return 2; }
  if (logm == 9) { lrs[0] = 4; return 1; }   // T = 32 (radix 8 would give T = 64)
  if (logm == 10) { lrs[0] = 3; return 1; }  // T = 128 (radix 16 would give T = 64)
  if (logm >= 12) { lrs[0] = 4; return 1; }
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
