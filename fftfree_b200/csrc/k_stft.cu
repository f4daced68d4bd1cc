// k_stft.cu -- launcher of the single-pass real-frame STFT kernels.
#include <cstdlib>

#include "fft_launch.cuh"

namespace ffb {
namespace {

// ------------------------------------------------------------------ staged frames
// The frames of one signal with full frames W = N, hop H a multiple of 4: a
// block's G consecutive frames cover the contiguous span of (G - 1) H + N
// samples, which one thread copies into shared memory with one bulk copy
// (cp.async.bulk, completion counted on an mbarrier), with the analysis
// window beside it; the groups then frame from shared memory instead of
// re-reading each sample N / H times through L1.  Each block copies for
// itself only, from this GPU's own buffer.  A block whose frames do not all lie inside the
// signal, or whose bounded wait for the copy gives up, loads from global
// memory as the other kernels do (the copy is then drained, bounded, before
// the block exits).

__device__ __forceinline__ uint32_t st_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool st_wait_parity(uint32_t bar, uint32_t parity, unsigned limit) {
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

__device__ __forceinline__ void st_bulk_load(void* dst, const void* src, unsigned bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   st_smem_addr(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
               : "memory");
}

// Shared memory of the staged kernel: the groups' tiles (rounded to 128
// bytes), the span, the window, the mbarrier.
template <class S>
__host__ __device__ constexpr size_t staged_tiles_bytes() {
  return (((size_t)Launch<S>::G * S::SMEM * sizeof(float2)) + 127) & ~(size_t)127;
}
template <class S>
size_t staged_smem_bytes(int H, bool win) {
  constexpr int G = Launch<S>::G, N = 2 * S::M;
  return staged_tiles_bytes<S>() + ((size_t)(G - 1) * H + N) * 4 + (win ? (size_t)N * 4 : 0) + 16;
}

template <class S, int MODE>
__global__ void __launch_bounds__(Launch<S>::BLOCK) k_stft_staged(StftIO<MODE> io, Twiddles tw) {
  extern __shared__ __align__(128) float2 smem[];
  constexpr int T = S::T, G = Launch<S>::G, M = S::M, N = 2 * M;
  constexpr unsigned kLimit = 1u << 22;  // try_wait polls before a block gives up
  const StftArgs& a = io.a;
  const int g = threadIdx.x / T;
  const int t = threadIdx.x - g * T;
  const long long f0 = (long long)blockIdx.x * G;
  const long long f = f0 + g;
  float2* sm = smem + g * S::SMEM;
  const int H = a.H;
  const unsigned span_n = (unsigned)((G - 1) * H + N);  // samples, a multiple of 4
  float* span = reinterpret_cast<float*>(reinterpret_cast<char*>(smem) + staged_tiles_bytes<S>());
  float* wst = span + span_n;
  uint64_t* bar = reinterpret_cast<uint64_t*>(wst + (a.win ? N : 0));
  const uint32_t bar_a = st_smem_addr(bar);
  // every frame of the block full and inside the signal (block-uniform)
  const bool staged = (f0 + G - 1) * (long long)H + N <= a.pcm_len;
  bool ok = false;
  if (staged) {
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned bytes = span_n * 4u + (a.win ? (unsigned)N * 4u : 0u);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
      st_bulk_load(span, a.pcm + f0 * H, span_n * 4u, bar_a);
      if (a.win) st_bulk_load(wst, a.win, (unsigned)N * 4u, bar_a);
    }
    ok = __syncthreads_and(st_wait_parity(bar_a, 0, kLimit));
  }
  float2 v[S::R];
  if (ok) {
    const float2* s2 = reinterpret_cast<const float2*>(span + g * H);  // g H even: 8-byte aligned
    const float2* w2 = reinterpret_cast<const float2*>(wst);
#pragma unroll
    for (int i = 0; i < S::R; ++i) {
      const int m = t + i * T;
      float2 z = s2[m];
      if (a.win) z = __fmul2_rn(z, w2[m]);
      v[i] = z;
    }
  } else {
    io.template load<S>(f, t, v, sm, tw);
  }
  fft_engine<S, GroupSync>(v, t, sm, tw);
  io.template store<S>(f, t, v, sm, tw);
  if (staged && !ok && threadIdx.x == 0) (void)st_wait_parity(bar_a, 0, 16u * kLimit);  // drain the copy
}

// FFTFREE_STFT_STAGED=1 selects the staged kernel where it applies (read at
// every call).  Off by default: on B200 it measured no faster than the plain
// kernel (STFT N=1024, H=256: 0.0602 against 0.0576 ms; N=2048, H=512
// magnitude: 0.1086 against 0.1087 ms): the frames then come from shared
// memory instead of L1 hits, and both are served by the same pipe, which
// bounds these kernels.
bool staged_wanted() {
  const char* e = std::getenv("FFTFREE_STFT_STAGED");
  return e && e[0] == '1';
}

template <class S, int MODE>
cudaError_t run_staged(const StftIO<MODE>& io, cudaStream_t st, uint64_t* launches) {
  using L = Launch<S>;
  const size_t smem = staged_smem_bytes<S>(io.a.H, io.a.win != nullptr);
  if (smem > 227 * 1024) return cudaErrorInvalidValue;
  if (smem > 48 * 1024) {
    const cudaError_t e =
        cudaFuncSetAttribute(k_stft_staged<S, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const long long grid = (io.a.frames + L::G - 1) / L::G;
  if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
  Twiddles tw{twiddle_pyramid(0, st), twiddle_pass_tables(st)};
  k_stft_staged<S, MODE><<<(unsigned)grid, L::BLOCK, smem, st>>>(io, tw);
  if (launches) ++*launches;
  return cudaGetLastError();
}

// The staged kernel for the default pass radix of real frames of 64 .. 4096
// samples; -1 where it does not apply (the caller takes the plain kernel).
template <int MODE>
cudaError_t try_staged(const StftArgs& a, int logm, int logr, cudaStream_t st, uint64_t* launches) {
  if (!staged_wanted() || a.mirror || a.inverse || a.sig_frames != 0 || a.W != a.N || a.N < 64 || a.N > 4096 ||
      (a.H & 3) || a.H <= 0 || (reinterpret_cast<uintptr_t>(a.pcm) & 15) ||
      (a.win && (reinterpret_cast<uintptr_t>(a.win) & 15)) || logr != choose_logr(logm, -1, true))
    return (cudaError_t)-1;
  const StftIO<MODE> io{a, ilog2i(a.N)};
  switch (logm) {
    case 5: return run_staged<Sched<5, 2>, MODE>(io, st, launches);
    case 6: return run_staged<Sched<6, 3>, MODE>(io, st, launches);
    case 7: return run_staged<Sched<7, 3>, MODE>(io, st, launches);
    case 8: return run_staged<Sched<8, 3>, MODE>(io, st, launches);
    case 9: return run_staged<Sched<9, 4>, MODE>(io, st, launches);
    case 10: return run_staged<Sched<10, 4>, MODE>(io, st, launches);
    case 11: return run_staged<Sched<11, 4>, MODE>(io, st, launches);
    default: return (cudaError_t)-1;
  }
}

}  // namespace

cudaError_t launch_stft(const StftArgs& a, int req_logr, cudaStream_t s, uint64_t* launches) {
  const int logm = (a.N == 1) ? 0 : ilog2i(a.N) - 1;
  const int logr = choose_logr(logm, req_logr, true);
  if (logr < 0) return cudaErrorInvalidValue;
  if (a.mag_only == 0 || a.mag_only == 1 || a.mag_only == 2) {
    cudaError_t e = (cudaError_t)-1;
    if (a.mag_only == 2) e = try_staged<4>(a, logm, logr, s, launches);
    else if (a.mag_only == 1) e = try_staged<3>(a, logm, logr, s, launches);
    else if (post_mode(a.pf) == 1) e = try_staged<1>(a, logm, logr, s, launches);
    else if (post_mode(a.pf) == 0) e = try_staged<0>(a, logm, logr, s, launches);
    if (e != (cudaError_t)-1) return e;
  }
  if (a.mag_only == 4) {
    if (post_mode(a.pf) != 0) return cudaErrorInvalidValue;
    return dispatch(StftIO<6>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  }
  if (a.mag_only == 3) return dispatch(StftIO<5>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  if (a.mag_only == 2) return dispatch(StftIO<4>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  if (a.mag_only) return dispatch(StftIO<3>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  switch (post_mode(a.pf)) {
    case 2: return dispatch(StftIO<2>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
    case 1: return dispatch(StftIO<1>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
    default: return dispatch(StftIO<0>{a, ilog2i(a.N)}, logm, logr, a.frames, s, launches);
  }
}

long long stft_loss_parts(long long frames, int N) { return frames * loss_slots(N / 2 > 0 ? N / 2 : 1); }

}  // namespace ffb
