// recovery.cpp -- dropout controls and the recovery coordinator.
//
// The reference injects test-only "worker crashes" (a thrown exception in a
// WorkerPool thread) and recovers by restoring the column range from a
// backup and retrying (eigen_fft.hpp:1176-1398), with a coordinator that
// splits persistently failing frame ranges in half (fft_cffi.cpp:826-1027).
// On a GPU nothing is allowed to fail on purpose, so this build takes every
// decision on the host: which range "drops", the restore-observer calls,
// the retry count and the splitting are reproduced; the transform itself
// always runs on the device, and frames the coordinator gives up on are
// rewritten with their restored input afterwards.
#include "recovery.h"

#include <algorithm>
#include <atomic>
#include <functional>
#include <mutex>
#include <random>
#include <thread>
#include <unordered_set>
#include <utility>

#include "../../include/fft_cffi.h"
#include "../../include/fftfree_b200.h"

namespace ffb {
namespace {

struct DropoutState {
  std::atomic<int> rate{0};
  std::atomic<int> period{0};
  std::atomic<int> on_len{0};
  std::atomic<int> phase{0};
  std::atomic<long long> single{-1};
  std::atomic<int> persistent{0};
  std::mutex m;
  std::unordered_set<size_t> dropped_once;
  DropoutState() {
    // WorkerPoolDebug::init_from_env (eigen_fft.hpp:132-141)
    if (const char* e = std::getenv("FFTFREE_DEBUG_DROPOUT_PCT")) {
      try {
        rate.store(std::clamp(std::stoi(e), 0, 100));
      } catch (...) {
      }
    }
  }
};

DropoutState& state() {
  static DropoutState s;
  return s;
}

std::mutex g_obs_mu;
fft_restore_observer_t g_observer = nullptr;

bool pattern_enabled() { return state().period.load() > 0 && state().on_len.load() > 0; }

// eigen_fft.hpp:1196-1234
bool decide_drop(size_t idx) {
  DropoutState& s = state();
  bool drop = false;
  const long long single = s.single.load();
  if (single >= 0 && (long long)idx == single) {
    drop = true;
  } else {
    const int period = s.period.load(), onlen = s.on_len.load(), phase = s.phase.load();
    if (period > 0 && onlen > 0) {
      const long long pos = (long long)idx + phase;
      const int mod = (int)((pos % period + period) % period);
      if (mod < onlen) drop = true;
    }
  }
  if (!drop) {
    const int rate = s.rate.load();
    if (rate > 0) {
      thread_local std::mt19937_64 rng((unsigned)std::hash<std::thread::id>()(std::this_thread::get_id()) ^
                                       0x9e3779b97f4a7c15ULL);
      std::uniform_int_distribution<int> dist(1, 100);
      if (dist(rng) <= rate) drop = true;
    }
  }
  if (drop && s.persistent.load() == 0) {
    std::lock_guard<std::mutex> g(s.m);
    if (s.dropped_once.count(idx)) drop = false;
    else s.dropped_once.insert(idx);
  }
  return drop;
}

void notify(size_t a, size_t b) {
  fft_restore_observer_t cb;
  {
    std::lock_guard<std::mutex> g(g_obs_mu);
    cb = g_observer;
  }
  if (cb) cb(a, b);
}

}  // namespace

size_t recovery_batch_frames(size_t N) {
  const size_t max_bytes = 64ull * 1024ull * 1024ull;
  const size_t per = N * 8;  // complex<float> column
  return std::max<size_t>(1, max_bytes / (per + 1));
}

void run_recovery_coordinator(size_t frames, std::vector<char>* raw) {
  constexpr int kRetryCount = 2;  // EIGFFT_JOB_RETRY_COUNT
  raw->assign(frames, 0);
  std::vector<std::pair<size_t, size_t>> cur;
  if (state().rate.load() > 0 || pattern_enabled() || state().single.load() >= 0) {
    for (size_t f = 0; f < frames; ++f) cur.emplace_back(f, f + 1);
  } else {
    cur.emplace_back(0, frames);
  }
  while (!cur.empty()) {
    std::vector<std::pair<size_t, size_t>> persistent;
    std::vector<int> restores(cur.size(), 0);
    for (size_t ri = 0; ri < cur.size(); ++ri) {
      const auto r = cur[ri];
      // pool worker loop, non-Windows variant (eigen_fft.hpp:1345-1398)
      int attempt = 0;
      for (;;) {
        if (!decide_drop(ri)) {
          for (size_t f = r.first; f < r.second; ++f) (*raw)[f] = 0;
          break;
        }
        // restore callback (fft_cffi.cpp:914-934)
        if (r.second > r.first) notify(r.first, r.second);
        for (size_t f = r.first; f < r.second; ++f) (*raw)[f] = 1;
        const int prev = restores[ri]++;
        if (prev + 1 >= kRetryCount) persistent.push_back(r);
        ++attempt;
        if (attempt > kRetryCount) break;
      }
    }
    if (persistent.empty()) break;
    std::vector<std::pair<size_t, size_t>> next;
    bool abort_batch = false;
    for (const auto& r : persistent) {
      const size_t len = r.second - r.first;
      if (len <= 1) {
        abort_batch = true;
        break;
      }
      const size_t mid = r.first + len / 2;
      next.emplace_back(r.first, mid);
      next.emplace_back(mid, r.second);
    }
    if (abort_batch) break;
    cur.swap(next);
  }
}

}  // namespace ffb

using namespace ffb;

extern "C" {

FFT_CFFI_API void fft_set_workerpool_debug_dropout(int pct) { state().rate.store(std::clamp(pct, 0, 100)); }

FFT_CFFI_API void fft_set_workerpool_dropout_pattern(int period, int on_len, int phase) {
  // WorkerPoolDebug::set_pattern (eigen_fft.hpp:143-150)
  if (period < 0) period = 0;
  if (on_len < 0) on_len = 0;
  if (period > 0 && on_len > period) on_len = period;
  state().period.store(period);
  state().on_len.store(on_len);
  state().phase.store(phase);
}

FFT_CFFI_API void fft_set_workerpool_dropout_single(long long index) { state().single.store(index); }

FFT_CFFI_API void fft_set_workerpool_dropout_persistent(int on) { state().persistent.store(on ? 1 : 0); }

FFT_CFFI_API void fft_clear_workerpool_dropout_history(void) {
  std::lock_guard<std::mutex> g(state().m);
  state().dropped_once.clear();
}

FFT_CFFI_API void fft_register_restore_observer(fft_restore_observer_t cb) {
  std::lock_guard<std::mutex> g(g_obs_mu);
  g_observer = cb;
}

FFT_CFFI_API size_t fftfree_debug_recovery_plan(size_t frames, char* raw_out) {
  std::vector<char> raw;
  run_recovery_coordinator(frames, &raw);
  size_t n = 0;
  for (size_t f = 0; f < frames; ++f) {
    if (raw_out) raw_out[f] = raw[f];
    n += raw[f] ? 1 : 0;
  }
  return n;
}

}  // extern "C"
