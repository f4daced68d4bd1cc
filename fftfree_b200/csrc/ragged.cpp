// ragged.cpp -- ragged batches of real transforms of mixed sizes and
// framings in one persistent launch: the work list, the per-size schedule
// autotuner and its on-disk cache, the CUDA graph of the launch, and the C
// ABI (fftfree_ragged_*).
//
// The reference has no ragged entry point: its callers create one context
// per transform size and framing and loop over the signals (fft_init_full +
// fft_execute_batched per size).  An item here gives the same outputs as
// fft_execute_batched with pad_mode 1 on a context (n_i, window W_i, hop H_i,
// transform = R2C, half_spectrum = 1, the item's analysis window,
// reduce_magnitude / store_polar as the plan's flags) for its signal.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <random>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fft_cffi.h"
#include "../../include/fftfree_b200.h"
#include "context.h"
#include "kernels.h"

namespace ffb {
namespace {

constexpr uint32_t kRaggedMagic = 0x52414744u;  // "RAGD"

struct RaggedPlan {
  uint32_t magic = kRaggedMagic;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<int> logm;               // per item (caller order): log2 of N/2
  std::vector<RaggedItem> items;       // per item (caller order)
  std::vector<long long> frames;       // per item
  std::vector<float> windows;          // analysis taps, items' win_off into it
  size_t samples = 0, bins = 0;
  PostFlags pf{};
  int lr[16] = {};                     // pass radix (log2) per log2 N/2 of the single-pass sizes
  int rounds[16] = {};                 // block-loads of frames per tile per log2 N/2 (0 read as 1)
  int grid = 0, ntiles = 0;
  DevBuf d_items, d_jobs, d_tiles, d_counter, d_scratch, d_windows, d_in, d_re, d_im, d_mag;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void* graph_ptrs[4] = {};
  uint64_t launches = 0;
  std::mutex mu;
};

RaggedPlan* as_plan(void* h) {
  auto* p = static_cast<RaggedPlan*>(h);
  return (p && p->magic == kRaggedMagic) ? p : nullptr;
}

#define RG_CHECK(expr)                                                                 \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess) {                                                           \
      std::fprintf(stderr, "[fftfree_b200] ragged: CUDA error %s at %s:%d\n",          \
                   cudaGetErrorName(_e), __FILE__, __LINE__);                          \
      throw std::runtime_error("cuda");                                                \
    }                                                                                  \
  } while (0)

int log2_exact(size_t v) {
  if (v == 0 || (v & (v - 1))) return -1;
  int l = 0;
  while ((size_t(1) << l) < v) ++l;
  return l;
}

bool is_device(const void* p) {
  cudaPointerAttributes at;
  if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------- work list
// Tiles of same-size frames in work order (largest sizes first); `only` >= 0
// restricts the list to one size (the tuner).
struct WorkList {
  std::vector<int4> tiles;
  std::vector<int2> jobs;
};

WorkList build_work(const RaggedPlan& p, int only) {
  WorkList w;
  std::vector<std::vector<int2>> by(ragged_max_log());
  for (size_t i = 0; i < p.logm.size(); ++i)
    for (long long f = 0; f < p.frames[i]; ++f) by[p.logm[i]].push_back(make_int2((int)i, (int)f));
  for (int L = ragged_max_log() - 1; L >= 0; --L) {
    if (by[L].empty() || (only >= 0 && L != only)) continue;
    const bool whole = ragged_block_log(L) != 0;
    const int T = std::max(1, (1 << L) >> p.lr[L]);
    const int per = whole ? 1 : std::max(1, ragged_block_threads() / T) * std::max(1, p.rounds[L]);
    for (size_t s = 0; s < by[L].size(); s += per) {
      const int n = (int)std::min<size_t>(per, by[L].size() - s);
      const int lr = (L == ragged_max_log() - 1) ? 0 : p.lr[L];
      w.tiles.push_back(make_int4((int)w.jobs.size(), n, L, lr));
      for (int k = 0; k < n; ++k) w.jobs.push_back(by[L][s + k]);
    }
  }
  return w;
}

void upload(RaggedPlan& p, const WorkList& w) {
  RG_CHECK(cudaMemcpyAsync(p.d_jobs.get(std::max<size_t>(1, w.jobs.size()) * sizeof(int2)), w.jobs.data(),
                           w.jobs.size() * sizeof(int2), cudaMemcpyHostToDevice, p.stream));
  RG_CHECK(cudaMemcpyAsync(p.d_tiles.get(std::max<size_t>(1, w.tiles.size()) * sizeof(int4)), w.tiles.data(),
                           w.tiles.size() * sizeof(int4), cudaMemcpyHostToDevice, p.stream));
  RG_CHECK(cudaStreamSynchronize(p.stream));
  p.ntiles = (int)w.tiles.size();
}

RaggedArgs args_for(RaggedPlan& p, const float* pcm, float* re, float* im, float* mag) {
  RaggedArgs a{};
  a.pcm = pcm;
  a.out_re = re;
  a.out_im = im;
  a.out_mag = mag;
  a.items = static_cast<const RaggedItem*>(p.d_items.p);
  a.jobs = static_cast<const int2*>(p.d_jobs.p);
  a.tiles = static_cast<const int4*>(p.d_tiles.p);
  a.ntiles = p.ntiles;
  a.counter = static_cast<int*>(p.d_counter.p);
  a.scratch = static_cast<float2*>(p.d_scratch.p);
  a.windows = static_cast<const float*>(p.d_windows.p);
  a.pf = p.pf;
  return a;
}

// ---------------------------------------------------------------- autotuner
// Cache of measured choices (pass radix and block-loads of frames per tile),
// keyed by (N, frames of that N, transform and kernel generation):
// FFTFREE_TUNE_CACHE names the file (default ~/.cache/fftfree_b200/tune.txt);
// FFTFREE_TUNE=0 turns tuning off (the default schedule of the size).
const char* const kTuneKind = "r2c.b1024.t";  // R2C on the 1024-thread persistent kernel, radix and tile
std::mutex g_cache_mu;
std::map<std::tuple<long long, long long, std::string>, std::pair<int, int>> g_cache;
bool g_cache_loaded = false;

std::string cache_path() {
  if (const char* e = std::getenv("FFTFREE_TUNE_CACHE")) return e;
  const char* home = std::getenv("HOME");
  return std::string(home ? home : ".") + "/.cache/fftfree_b200/tune.txt";
}

void cache_load() {
  if (g_cache_loaded) return;
  g_cache_loaded = true;
  std::ifstream f(cache_path());
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream s(line);
    std::string kind, tr;
    long long n = 0, batch = 0;
    int lr = 0, rounds = 0;
    if (s >> kind >> tr >> n >> batch >> lr >> rounds && kind == "ragged" && lr >= 2 && lr <= 5 && rounds >= 1 &&
        rounds <= 8)
      g_cache[{n, batch, tr}] = {lr, rounds};
  }
}

void cache_store(long long n, long long batch, const std::string& tr, int lr, int rounds) {
  g_cache[{n, batch, tr}] = {lr, rounds};
  const std::string path = cache_path();
  const size_t slash = path.find_last_of('/');
  if (slash != std::string::npos) {
    // create the cache folder, one level at a time
    const std::string dir = path.substr(0, slash);
    for (size_t i = 1; i <= dir.size(); ++i)
      if (i == dir.size() || dir[i] == '/') (void)mkdir(dir.substr(0, i).c_str(), 0755);
  }
  std::ofstream f(path, std::ios::app);
  if (f) f << "ragged " << tr << " " << n << " " << batch << " " << lr << " " << rounds << "\n";
}

bool tuning_on() {
  const char* e = std::getenv("FFTFREE_TUNE");
  return !(e && e[0] == '0');
}

float time_launch(RaggedPlan& p, const RaggedArgs& a) {
  cudaEvent_t e0, e1;
  RG_CHECK(cudaEventCreate(&e0));
  RG_CHECK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    RG_CHECK(cudaMemsetAsync(a.counter, 0, sizeof(int), p.stream));
    RG_CHECK(cudaEventRecord(e0, p.stream));
    RG_CHECK(launch_ragged(a, p.grid, p.stream, &p.launches));
    RG_CHECK(cudaEventRecord(e1, p.stream));
    RG_CHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    RG_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best = std::min(best, ms);  // the first one warms up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

// Per size, largest first: the pass radix among the size's candidates and
// the tile size (1, 2 or 4 block-loads of frames per claimed tile: more per
// tile claims fewer tiles, fewer per tile balances the blocks' last tiles
// better).  Each pair is timed on the whole launch of the plan's work list
// (the other sizes at their choices so far), since sizes share the
// persistent blocks; a pair replaces the current choice only when it is at
// least 0.5% faster.  The samples are uniform in [-1, 1), not the caller's.
// The tuner's samples: uniform in [-1, 1) (a fixed std::mt19937 draw of up
// to 2^20 floats, repeated), so that its timings see the arithmetic of real
// spectra (all-zero frames would take the magnitude's small-value path).
void fill_tuner_input(RaggedPlan& p) {
  const size_t n = std::max<size_t>(1, p.samples);
  float* d = static_cast<float*>(p.d_in.get(n * 4));
  const size_t m = std::min<size_t>(n, (size_t)1 << 20);
  std::vector<float> h(m);
  std::mt19937 gen(7);
  std::uniform_real_distribution<float> u(-1.0f, 1.0f);
  for (auto& v : h) v = u(gen);
  RG_CHECK(cudaMemcpyAsync(d, h.data(), m * 4, cudaMemcpyHostToDevice, p.stream));
  for (size_t done = m; done < n;) {  // doubling device copies
    const size_t c = std::min(done, n - done);
    RG_CHECK(cudaMemcpyAsync(d + done, d, c * 4, cudaMemcpyDeviceToDevice, p.stream));
    done += c;
  }
  RG_CHECK(cudaStreamSynchronize(p.stream));  // the host draw is released on return
}

void tune(RaggedPlan& p) {
  std::vector<long long> count(ragged_max_log(), 0);
  for (size_t i = 0; i < p.logm.size(); ++i) count[p.logm[i]] += p.frames[i];
  std::lock_guard<std::mutex> lk(g_cache_mu);
  cache_load();
  for (int L = 0; L < ragged_max_log(); ++L) {
    int cand[4];
    const int nc = ragged_candidates(L, cand);
    p.rounds[L] = 1;
    if (!count[L] || nc == 0) continue;
    // default: the single-pass kernels' choice for real input, within the candidates
    int def = choose_logr(L, -1, true);
    if (std::find(cand, cand + nc, def) == cand + nc) def = cand[nc - 1];
    p.lr[L] = def;
    // tile sizes worth trying: only while the size has frames for more than
    // one block-load per tile (whole-block sizes take one frame per tile)
    std::vector<int> rounds_c{1};
    if (ragged_block_log(L) == 0) {
      const long long per = std::max(1, ragged_block_threads() / std::max(1, (1 << L) >> def));
      for (int r : {2, 4})
        if (count[L] > per * r) rounds_c.push_back(r);
    }
    if ((nc == 1 && rounds_c.size() == 1) || !tuning_on()) continue;
    const long long n = 2LL << L;
    auto it = g_cache.find({n, count[L], kTuneKind});
    if (it != g_cache.end() && std::find(cand, cand + nc, it->second.first) != cand + nc) {
      p.lr[L] = it->second.first;
      p.rounds[L] = it->second.second;
      continue;
    }
    const auto time_with = [&](int lr, int r) {
      p.lr[L] = lr;
      p.rounds[L] = r;
      upload(p, build_work(p, -1));
      const RaggedArgs a = args_for(p, static_cast<const float*>(p.d_in.p), static_cast<float*>(p.d_re.p),
                                    static_cast<float*>(p.d_im.p), static_cast<float*>(p.d_mag.p));
      return time_launch(p, a);
    };
    int pick = def, pick_rounds = 1;
    float best = time_with(def, 1);
    for (int c = 0; c < nc; ++c) {
      for (int r : rounds_c) {
        if (cand[c] == def && r == 1) continue;
        const float ms = time_with(cand[c], r);
        if (ms < 0.995f * best) {
          best = ms;
          pick = cand[c];
          pick_rounds = r;
        }
      }
    }
    p.lr[L] = pick;
    p.rounds[L] = pick_rounds;
    cache_store(n, count[L], kTuneKind, pick, pick_rounds);
  }
}

// ---------------------------------------------------------------- graph
void capture(RaggedPlan& p, const float* pcm, float* re, float* im, float* mag) {
  const void* key[4] = {pcm, re, im, mag};
  if (p.exec && std::equal(key, key + 4, p.graph_ptrs)) return;
  if (p.exec) {
    cudaGraphExecDestroy(p.exec);
    cudaGraphDestroy(p.graph);
    p.exec = nullptr;
    p.graph = nullptr;
  }
  const RaggedArgs a = args_for(p, pcm, re, im, mag);
  RG_CHECK(cudaStreamBeginCapture(p.stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e1 = cudaMemsetAsync(a.counter, 0, sizeof(int), p.stream);
  cudaError_t e2 = (e1 == cudaSuccess) ? launch_ragged(a, p.grid, p.stream, nullptr) : e1;
  cudaGraph_t g = nullptr;
  const cudaError_t e3 = cudaStreamEndCapture(p.stream, &g);
  RG_CHECK(e1);
  RG_CHECK(e2);
  RG_CHECK(e3);
  p.graph = g;
  RG_CHECK(cudaGraphInstantiate(&p.exec, g, 0));
  std::copy(key, key + 4, p.graph_ptrs);
}

struct Guard {
  int prev = -1;
  explicit Guard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~Guard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" {

FFT_CFFI_API void* fftfree_ragged_plan_stft(const size_t* n, const size_t* lengths, const int* window,
                                            const int* hop, const int* window_kind, const float* window_param,
                                            size_t count, int reduce_magnitude, int store_polar) {
  if (!n || !lengths || count == 0 || count > (size_t)1 << 30) return nullptr;
  RaggedPlan* p = nullptr;
  try {
    p = new RaggedPlan();
    RG_CHECK(cudaGetDevice(&p->device));
    p->logm.resize(count);
    p->items.resize(count);
    p->frames.resize(count);
    std::map<std::tuple<int, int, float>, int> taps;  // (kind, W, p1) -> offset in windows
    size_t jobs = 0;
    for (size_t i = 0; i < count; ++i) {
      const int lg = log2_exact(n[i]);
      const int N = (int)n[i];
      const int W = (window && window[i] > 0) ? window[i] : N;
      const int H = (hop && hop[i] > 0) ? hop[i] : W;
      if (lg < 2 || lg > ragged_max_log() || W > N || H <= 0 || lengths[i] > ((size_t)1 << 40)) {
        std::fprintf(stderr, "[fftfree_b200] fftfree_ragged_plan: item %zu: n = %zu must be a power of two in "
                             "[4, %d], window <= n, hop > 0\n", i, n[i], 1 << ragged_max_log());
        delete p;
        return nullptr;
      }
      RaggedItem& it = p->items[i];
      it.pcm_off = (long long)p->samples;
      it.pcm_len = (long long)lengths[i];
      it.out_off = (long long)p->bins;
      it.W = W;
      it.H = H;
      it.win_off = -1;
      const int kind = window_kind ? window_kind[i] : 0;
      const float p1 = window_param ? window_param[i] : 0.f;
      if (kind != FFT_WINDOW_RECT) {
        auto key = std::make_tuple(kind, W, p1);
        auto f = taps.find(key);
        if (f == taps.end()) {
          // taps 4-float aligned, so the 8-byte loads of a frame stay aligned
          while (p->windows.size() % 4) p->windows.push_back(0.f);
          const std::vector<float> w = window_taps(kind, W, p1, 0.f, FFT_WINDOW_NORM_NONE);
          f = taps.emplace(key, (int)p->windows.size()).first;
          p->windows.insert(p->windows.end(), w.begin(), w.end());
        }
        it.win_off = f->second;
      }
      // frames of fft_execute_batched with pad_mode 1 (fft_cffi.cpp:710-750)
      long long fr = 0;
      if (lengths[i] > 0) fr = (lengths[i] < (size_t)W) ? 1 : 1 + (long long)((lengths[i] - W) / H);
      p->logm[i] = lg - 1;
      p->frames[i] = fr;
      p->samples += lengths[i];
      p->bins += (size_t)fr * (n[i] / 2 + 1);
      jobs += (size_t)fr;
    }
    if (jobs > (size_t)0x7fffffff) throw std::runtime_error("too many frames");
    p->pf.r2c_half = 1;
    p->pf.polar = store_polar ? 1 : 0;
    p->pf.reduce = (!store_polar && reduce_magnitude) ? 1 : 0;
    RG_CHECK(cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking));
    p->stream = p->own_stream;
    (void)twiddle_pyramid(ragged_max_log(), p->stream);  // built before any capture
    if (!twiddle_pass_tables(p->stream)) throw std::runtime_error("twiddle tables");
    p->grid = ragged_grid();
    p->d_counter.get(sizeof(int));
    RG_CHECK(cudaMemcpyAsync(p->d_items.get(count * sizeof(RaggedItem)), p->items.data(),
                             count * sizeof(RaggedItem), cudaMemcpyHostToDevice, p->stream));
    if (!p->windows.empty())
      RG_CHECK(cudaMemcpyAsync(p->d_windows.get(p->windows.size() * 4), p->windows.data(), p->windows.size() * 4,
                               cudaMemcpyHostToDevice, p->stream));
    bool any_split = false;
    for (size_t i = 0; i < count; ++i) any_split = any_split || (p->logm[i] == ragged_max_log() - 1 && p->frames[i]);
    if (any_split) p->d_scratch.get((size_t)p->grid * ragged_scratch_per_block());
    // staging (host buffers) and the tuner's buffers
    fill_tuner_input(*p);
    p->d_re.get(std::max<size_t>(1, p->bins) * 4);
    p->d_im.get(std::max<size_t>(1, p->bins) * 4);
    p->d_mag.get(std::max<size_t>(1, p->bins) * 4);
    tune(*p);
    upload(*p, build_work(*p, -1));
    return p;
  } catch (...) {
    delete p;
    return nullptr;
  }
}

FFT_CFFI_API void* fftfree_ragged_plan(const size_t* sizes, size_t count, int reduce_magnitude,
                                       int store_polar) {
  // one frame per item: window = hop = the item's size, no window taps
  return fftfree_ragged_plan_stft(sizes, sizes, nullptr, nullptr, nullptr, nullptr, count, reduce_magnitude,
                                  store_polar);
}

FFT_CFFI_API size_t fftfree_ragged_frames(void* plan, size_t item) {
  RaggedPlan* p = as_plan(plan);
  return (p && item < p->frames.size()) ? (size_t)p->frames[item] : 0;
}

FFT_CFFI_API size_t fftfree_ragged_samples(void* plan) {
  RaggedPlan* p = as_plan(plan);
  return p ? p->samples : 0;
}

FFT_CFFI_API size_t fftfree_ragged_bins(void* plan) {
  RaggedPlan* p = as_plan(plan);
  return p ? p->bins : 0;
}

FFT_CFFI_API int fftfree_ragged_schedule(void* plan, size_t n) {
  RaggedPlan* p = as_plan(plan);
  const int lg = log2_exact(n);
  if (!p || lg < 2 || lg > ragged_max_log()) return 0;
  return (lg - 1 == ragged_max_log() - 1) ? 0 : (1 << p->lr[lg - 1]);
}

FFT_CFFI_API int fftfree_ragged_tile(void* plan, size_t n) {
  RaggedPlan* p = as_plan(plan);
  const int lg = log2_exact(n);
  if (!p || lg < 2 || lg > ragged_max_log()) return 0;
  const int L = lg - 1;
  if (ragged_block_log(L) != 0) return 1;
  const int T = std::max(1, (1 << L) >> p->lr[L]);
  return std::max(1, ragged_block_threads() / T) * std::max(1, p->rounds[L]);
}

FFT_CFFI_API void fftfree_ragged_set_stream(void* plan, void* stream) {
  RaggedPlan* p = as_plan(plan);
  if (!p) return;
  std::lock_guard<std::mutex> lk(p->mu);
  p->stream = stream ? static_cast<cudaStream_t>(stream) : p->own_stream;
}

FFT_CFFI_API int fftfree_ragged_execute(void* plan, const float* pcm, float* out_real, float* out_imag,
                                        float* out_mag) {
  RaggedPlan* p = as_plan(plan);
  if (!p || !pcm || !out_real || !out_imag || !out_mag) return 0;
  try {
    std::lock_guard<std::mutex> lk(p->mu);
    Guard g(p->device);
    const bool in_host = !is_device(pcm);
    float* outs[3] = {out_real, out_imag, out_mag};
    DevBuf* stage[3] = {&p->d_re, &p->d_im, &p->d_mag};
    float* dev_out[3];
    bool out_host[3];
    for (int k = 0; k < 3; ++k) {
      out_host[k] = !is_device(outs[k]);
      dev_out[k] = out_host[k] ? static_cast<float*>(stage[k]->p) : outs[k];
    }
    const float* d_pcm = pcm;
    if (in_host) {
      RG_CHECK(cudaMemcpyAsync(p->d_in.p, pcm, p->samples * 4, cudaMemcpyHostToDevice, p->stream));
      d_pcm = static_cast<const float*>(p->d_in.p);
    }
    capture(*p, d_pcm, dev_out[0], dev_out[1], dev_out[2]);
    RG_CHECK(cudaGraphLaunch(p->exec, p->stream));
    ++p->launches;
    bool any_host = in_host;
    for (int k = 0; k < 3; ++k)
      if (out_host[k]) {
        RG_CHECK(cudaMemcpyAsync(outs[k], dev_out[k], p->bins * 4, cudaMemcpyDeviceToHost, p->stream));
        any_host = true;
      }
    if (any_host) RG_CHECK(cudaStreamSynchronize(p->stream));
    return 1;
  } catch (...) {
    return 0;
  }
}

FFT_CFFI_API unsigned long long fftfree_ragged_launch_count(void* plan) {
  RaggedPlan* p = as_plan(plan);
  return p ? p->launches : 0;
}

FFT_CFFI_API void fftfree_ragged_free(void* plan) {
  RaggedPlan* p = as_plan(plan);
  if (!p) return;
  {
    Guard g(p->device);
    cudaStreamSynchronize(p->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->own_stream) cudaStreamDestroy(p->own_stream);
    p->magic = 0;
  }
  delete p;
}

}  // extern "C"
