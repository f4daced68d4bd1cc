// k_ragged.cu -- one persistent launch over a ragged batch of real
// transforms (R2C, half spectrum) of different sizes and framings.
//
// Item i is a signal framed as fft_execute_batched frames it (pad_mode 1,
// fft_cffi.cpp:701-824): frames of W_i samples at hop H_i, zero-padded to
// N_i, windowed by the item's analysis taps; its frames' planar (re, im,
// mag) rows of N_i/2 + 1 bins are concatenated in item order.  Every frame
// is one job; the host groups the jobs of one size into tiles, largest
// first (longest processing time first balances the persistent blocks), and
// the blocks (512 threads, two per SM, so that one block's loads overlap the
// other's transforms) take tiles from an atomic counter until the list is
// exhausted.  A tile is
//  * a group of same-size frames of up to 2^13 complex points, one per
//    T-thread slice of the block -- the single-pass engine and the STFT
//    load / store policy of fft_execute_batched, so a frame matches that
//    call bit for bit where the radix is the same;
//  * one frame of 2^14 or 2^15 complex points (N = 32768, 65536), beyond one
//    block's shared memory: a decimation-in-time split into P = 2 or 4
//    transforms of 2^13 points run one after the other through the block's
//    engine, the frame read once, the pending points and spectra in a
//    scratch slot of the block (2^15 points, 256 KB; 296 slots, 76 MB:
//    L2-resident), and a combine step that untangles bins k + (M/P) j for all
//    j together so that the outputs stay contiguous.
#include "fft_launch.cuh"

namespace ffb {
namespace {

constexpr int kBlock = 512;
constexpr int kSubLog = 13;    // log2 complex points of one block's single pass
constexpr int kMaxLog = 15;    // log2 complex points of the largest item

// ---------------------------------------------------------------- single-pass tile
template <class S, int MODE>
__device__ __forceinline__ void ragged_single(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
  constexpr int T = S::T;
  static_assert(T <= 32 || kBlock / T <= 15 || T >= 256, "named barrier per group");
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  const bool ok = g < tile.y;
  const int2 job = __ldg(a.jobs + tile.x + (ok ? g : 0));
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
  float2* sm = smem + g * S::SMEM;
  float2 v[S::R];
  io.template load<S>(job.y, t, v, sm, tw);
  fft_engine<S, GroupSync>(v, t, sm, tw);
  io.template store<S>(job.y, t, v, sm, tw);
}

// ---------------------------------------------------------------- split tile
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

// exp(-2 pi i q / P) for q < P (P = 2 or 4): 1, -1 / 1, -i, -1, i.
template <int P>
__device__ __forceinline__ float2 root_p(int q) {
  if constexpr (P == 2) return make_float2(q ? -1.f : 1.f, 0.f);
  return wconst<4>(q);
}

// M = P * 2^13 complex points z[m] = (s[2m], s[2m+1]) of an N = 2M frame, by
// decimation in time: E_q = DFT_{M/P}(z[P n + q]), then for k < M/P
//   Z[k + (M/P) j] = sum_q exp(-2 pi i q j / P) w_M^(q k) E_q[k],
// and X[k + (M/P) j] = untangle(Z[k + (M/P) j], Z[M - k - (M/P) j]).  The frame is
// read once (the P points z[P n .. P n + P - 1] of each n together): z[P n]
// stays in registers for the first transform, the others wait in the block's
// scratch slot (M points) and are transformed there in place; the last
// spectrum goes to the tile.  The combine reads E_q at k and M/P - k and
// writes bins k + (M/P) j for every j: contiguous across the block's lanes.
template <int P, class S>
__device__ __forceinline__ void split_frame(const RaggedArgs& a, int4 tile, const float** src, const float** win,
                                            long long* cnt, bool* fast) {
  const int2 job = __ldg(a.jobs + tile.x);
  const RaggedItem it = a.items[job.x];
  *src = stft_frame(a.pcm + it.pcm_off, it.pcm_len, 0, 0, it.W, it.H, job.y, cnt);
  *win = it.win_off >= 0 ? a.windows + it.win_off : nullptr;
  *fast = *cnt == 2LL * P * S::M && aligned8(*src) && (!*win || aligned8(*win));
}

template <int P, int MODE>
__device__ __forceinline__ void ragged_split(const RaggedArgs& a, int4 tile, float2* smem, const Twiddles& tw) {
  using S = Sched<kSubLog, 4>;
  constexpr int T = S::T, R = S::R, MQ = S::M, M = P * MQ, LM = kSubLog + (P == 2 ? 1 : 2);
  static_assert(T == kBlock, "the whole block per sub-transform");
  const int t = threadIdx.x;
  float2* scr = a.scratch + (long long)blockIdx.x * (1LL << kMaxLog);  // the block's slot (the largest size)
  // sub-transform q: the first reads the frame once -- z[P n] into the
  // registers, z[P n + q'] (q' > 0) into slot q' -- the others their slot
  // (each thread reads only its own points before the engine's first
  // barrier); spectra back into the slots, the last one into the tile.  One
  // engine body for all of them (a second copy would keep the first one's
  // address arithmetic live, beyond the register budget).
#pragma unroll 1
  for (int q = 0; q < P; ++q) {
    float2 v[R];
    if (q == 0) {
      const float* src;
      const float* win;
      long long cnt;
      bool fast;
      split_frame<P, S>(a, tile, &src, &win, &cnt, &fast);
#pragma unroll
      for (int i = 0; i < R; ++i) {
        const int n = t + i * T;
#pragma unroll
        for (int qq = 0; qq < P; ++qq) {
          const float2 z = frame_pair(src, win, cnt, 2LL * (P * (long long)n + qq), fast);
          if (qq == 0) v[i] = z;
          else scr[qq * MQ + n] = z;
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < R; ++i) v[i] = scr[q * MQ + t + i * T];
    }
    fft_engine<S, GroupSync>(v, t, smem, tw);
    if (q == P - 1) {
      tile_write_natural<S>(v, t, smem);
    } else {
#pragma unroll
      for (int i = 0; i < R; ++i) scr[q * MQ + t + i * T] = v[i];
    }
  }
  __syncthreads();

  const int2 job = __ldg(a.jobs + tile.x);
  const RaggedItem it = a.items[job.x];
  StftArgs sa{};
  sa.N = 2 * M;
  sa.pf = a.pf;
  sa.mag_from_real = 1;
  const StftIO<MODE> io{sa, LM + 1};
  const bool mag_is_re = (MODE == 1) || (MODE == 2);
  float* re = a.out_re + it.out_off + (long long)job.y * (M + 1);
  float* im = a.out_im + it.out_off + (long long)job.y * (M + 1);
  float* mg = a.out_mag + it.out_off + (long long)job.y * (M + 1);
  // E_q of bin k: the last one from the tile, the others from their slots
  const auto E = [&](int q, int k) -> float2 { return q == P - 1 ? smem[pidx(k)] : scr[q * MQ + k]; };
#pragma unroll 1
  for (int i = 0; i < R; ++i) {
    const int k = t + i * T;
    float2 A[P], B[P];
    float2 wq[P];  // w_M^(q k)
#pragma unroll
    for (int q = 0; q < P; ++q) {
      wq[q] = q ? tw_get(tw, LM, (unsigned)(q * k)) : make_float2(1.f, 0.f);
      A[q] = q ? cmul(E(q, k), wq[q]) : E(0, k);
    }
    if constexpr (P == 2) {
      Dft<2>::run(A);
    } else {
      Dft<4>::run(A);
    }
    if (k > 0) {
      // w_M^(q (M/P - k)) = exp(-2 pi i q / P) conj(w_M^(q k))
#pragma unroll
      for (int q = 0; q < P; ++q)
        B[q] = q ? cmul(E(q, MQ - k), cmul(root_p<P>(q), cconj(wq[q]))) : E(0, MQ - k);
      if constexpr (P == 2) {
        Dft<2>::run(B);
      } else {
        Dft<4>::run(B);
      }
    }
    const float2 wn = tw_get(tw, LM + 1, (unsigned)k);  // w_N^k
#pragma unroll
    for (int j = 0; j < P; ++j) {
      // partner Z[M - k - (M/P) j]: B[P-1-j] (k > 0), A[(P - j) mod P] (k = 0)
      const float2 zm = k ? B[P - 1 - j] : A[(P - j) & (P - 1)];
      const float2 c = wconst<2 * P>(j);  // w_N^((M/P) j)
      const float2 h = make_float2(0.5f * (wn.x * c.x - wn.y * c.y), 0.5f * (wn.x * c.y + wn.y * c.x));
      float2 X = untangle_bin(A[j], zm, h);
      if (k == 0 && j == 0) X.y = 0.f;  // DC
      io.emit(re, im, mg, k + MQ * j, X, k == 0 && j == 0, 1.0f, mag_is_re);
    }
    if (k == 0) io.emit(re, im, mg, M, make_float2(A[0].x - A[0].y, 0.f), true, 1.0f, mag_is_re);  // Nyquist
  }
  __syncthreads();  // shared memory and scratch are reused by the block's next tile
}

// ---------------------------------------------------------------- dispatch
// tile.z = log2 complex points, tile.w = pass radix (log2), 0 for the split
// paths; the pass radices keep T = M / R <= 32 or >= 64 (named barriers per
// group: 8 at most in a 512-thread block).
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
    FFB_RS(11, 3) FFB_RS(11, 4) FFB_RS(12, 3) FFB_RS(12, 4) FFB_RS(13, 4)
    case (kSubLog + 1) * 8: ragged_split<2, MODE>(a, tile, smem, tw); return;
    case (kSubLog + 2) * 8: ragged_split<4, MODE>(a, tile, smem, tw); return;
    default: return;
  }
#undef FFB_RS
}

template <int MODE>
__global__ void __launch_bounds__(kBlock, 2) k_ragged(RaggedArgs a, Twiddles tw) {
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
  // padding per point: 128 groups of 64 points take the most)
  return cmax(cmax(cmax(cmax(tile_smem<1, 2>(), tile_smem<2, 2>()), cmax(tile_smem<3, 2>(), tile_smem<4, 2>())),
                   cmax(cmax(tile_smem<5, 2>(), tile_smem<5, 3>()), cmax(tile_smem<6, 3>(), tile_smem<6, 4>()))),
              cmax(cmax(cmax(tile_smem<7, 3>(), tile_smem<7, 4>()), cmax(tile_smem<8, 3>(), tile_smem<8, 4>())),
                   cmax(cmax(cmax(tile_smem<9, 3>(), tile_smem<9, 4>()), cmax(tile_smem<10, 3>(), tile_smem<10, 4>())),
                        cmax(cmax(tile_smem<11, 3>(), tile_smem<11, 4>()),
                             cmax(cmax(tile_smem<12, 3>(), tile_smem<12, 4>()), tile_smem<13, 4>())))));
}
static_assert(2 * ragged_smem_bytes() <= 226 * 1024, "two blocks per SM");

template <int MODE>
cudaError_t launch_mode(const RaggedArgs& a, int grid, cudaStream_t st, uint64_t* launches) {
  const size_t smem = ragged_smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(k_ragged<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  Twiddles tw{twiddle_pyramid(kMaxLog + 1, st), twiddle_pass_tables(st)};
  k_ragged<MODE><<<grid, kBlock, smem, st>>>(a, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

}  // namespace

int ragged_max_log() { return kMaxLog + 1; }  // log2 N of the largest item
int ragged_block_log(int logm) { return logm > kSubLog ? 1 : 0; }
size_t ragged_scratch_per_block() { return (size_t)(1u << kMaxLog) * sizeof(float2); }
int ragged_block_threads() { return kBlock; }

int ragged_candidates(int logm, int* lrs) {
  if (logm > kSubLog) return 0;
  if (logm <= 4) { lrs[0] = 2; return 1; }
  if (logm == 5) { lrs[0] = 2; lrs[1] = 3; return 2; }
  if (logm == kSubLog) { lrs[0] = 4; return 1; }  // T = 512, the whole block
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
