// TEST INFRASTRUCTURE ONLY: a C entry to the reference's own C++ batched
// transform, eigfft::fft_inplace_batched_with_metadata
// (eigen_fft.hpp:3152-3168), so that tests and the CPU baseline can run the
// reference's executors on complex batches (its C ABI has no complex-output
// entry).  It is compiled together with the unchanged reference sources into
// oracle/_ref/ by oracle/Makefile and is never linked into the product.
//
// The plan is set up the way the reference's C ABI sets up its shared plan
// (fft_cffi.cpp:792-806): PlanEnvironment::initialize with a
// PlanRuntimeConfig (plan_support.hpp:24-45, 57-174), the kernel chosen with
// Plan::use_kernel (1 = Cooley-Tukey, 2 = Stockham, otherwise the plan's
// default), and a dispatcher that forwards to a WorkerPool of `threads`
// threads (the PoolDispatcher of fft_cffi.cpp:284-310).
#include <Eigen/Core>

#include <complex>
#include <cstddef>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "eigen_fft.hpp"
#include "fft_cffi.hpp"
#include "plan_support.hpp"

namespace {

struct RefPoolDispatcher : public eigfft::JobDispatcher {
  eigfft::WorkerPool* pool = nullptr;
  void parallel_for(size_t total, size_t chunk, const Fn& fn) override {
    if (!pool || total == 0) {
      eigfft::InlineDispatcher::instance().parallel_for(total, chunk, fn);
      return;
    }
    pool->parallel_for(total, chunk == 0 ? 1 : chunk, fn);
  }
  void parallel_for_with_restore(size_t total, size_t chunk, const Fn& fn,
                                 std::function<void(size_t, size_t)> restore_fn, eigfft::RecoveryOps ops,
                                 void* job_ctx) override {
    if (!pool || total == 0) {
      eigfft::InlineDispatcher::instance().parallel_for_with_restore(total, chunk, fn, std::move(restore_fn), ops,
                                                                      job_ctx);
      return;
    }
    pool->parallel_for_with_restore_ex(total, chunk == 0 ? 1 : chunk, fn, std::move(restore_fn), ops, job_ctx);
  }
};

// Restore-observer calls recorded in C: the reference invokes the observer
// from its WorkerPool threads (fft_cffi.cpp:315-319, eigen_fft.hpp:1290-1300),
// where a Python callback would add interpreter locking to the timing of the
// recovery path.
std::mutex g_obs_mu;
std::vector<std::pair<size_t, size_t>> g_obs;

void record_restore(size_t start, size_t end) {
  std::lock_guard<std::mutex> lock(g_obs_mu);
  g_obs.emplace_back(start, end);
}

struct RefPlan {
  eigfft::PlanEnvironment<float> env;
  std::unique_ptr<eigfft::WorkerPool> pool;
  RefPoolDispatcher dispatcher;
};

}  // namespace

extern "C" {

struct ref_meta_req {
  int kind;        // eigfft::MetadataKind value (eigen_fft.hpp:1477-1491)
  float* buf;      // `count` interleaved complex floats
  size_t count;
};

// A plan of N points with the context options that shape results; threads
// > 1 runs the batch on a WorkerPool.  Returns NULL on failure.
__attribute__((visibility("default"))) void* ref_plan_create(int N, int inverse, int kernel, int transform,
                                                             int reduce_magnitude, int store_polar,
                                                             int half_spectrum, int threads) {
  try {
    auto* p = new RefPlan();
    eigfft::PlanRuntimeConfig cfg;
    cfg.threads = threads < 1 ? 1 : threads;
    cfg.lanes = 1;
    cfg.inverse = inverse != 0;
    cfg.transform = transform;
    cfg.reduce_magnitude = reduce_magnitude != 0;
    cfg.store_polar = store_polar != 0;
    cfg.half_spectrum = half_spectrum != 0;
    p->env.initialize(N, inverse != 0, cfg);
    auto& plan = p->env.plan();
    if (kernel == 1) plan.use_kernel(eigfft::KernelKind::CooleyTukey);
    else if (kernel == 2) plan.use_kernel(eigfft::KernelKind::Stockham);
    if (cfg.threads > 1) {
      p->pool = std::make_unique<eigfft::WorkerPool>(cfg.threads);
      p->dispatcher.pool = p->pool.get();
      plan.set_dispatcher(&p->dispatcher);
    }
    return p;
  } catch (...) {
    return nullptr;
  }
}

// In-place transform of `batch` columns of N complex floats (column-major,
// column = transform), with optional metadata requests.  Returns 1 on
// success, 0 when the reference threw.
__attribute__((visibility("default"))) int ref_plan_execute(void* h, float* X, size_t batch,
                                                            const ref_meta_req* reqs, int nreq) {
  if (!h || !X) return 0;
  try {
    auto* p = static_cast<RefPlan*>(h);
    auto& plan = p->env.plan();
    std::vector<eigfft::MetadataRequest<float>> mr(static_cast<size_t>(nreq > 0 ? nreq : 0));
    for (int i = 0; i < nreq; ++i) {
      mr[i].kind = static_cast<eigfft::MetadataKind>(reqs[i].kind);
      mr[i].complex_buffer = reinterpret_cast<std::complex<float>*>(reqs[i].buf);
      mr[i].element_count = reqs[i].count;
    }
    Eigen::Map<Eigen::Matrix<std::complex<float>, Eigen::Dynamic, Eigen::Dynamic, Eigen::ColMajor>> m(
        reinterpret_cast<std::complex<float>*>(X), static_cast<Eigen::Index>(plan.N),
        static_cast<Eigen::Index>(batch));
    eigfft::fft_inplace_batched_with_metadata<float>(m, plan, mr.empty() ? nullptr : mr.data(),
                                                     static_cast<int>(mr.size()));
    return 1;
  } catch (...) {
    return 0;
  }
}

__attribute__((visibility("default"))) void ref_plan_free(void* h) {
  auto* p = static_cast<RefPlan*>(h);
  if (!p) return;
  if (p->pool) p->env.plan().set_dispatcher(nullptr);
  delete p;
}

// Registers the recording observer (fft_register_restore_observer) and
// clears the record.
__attribute__((visibility("default"))) void ref_observer_attach(void) {
  {
    std::lock_guard<std::mutex> lock(g_obs_mu);
    g_obs.clear();
  }
  fft_register_restore_observer(&record_restore);
}

// Copies up to `cap` recorded (start, end) pairs into out[2 * i], out[2 * i + 1];
// returns how many were recorded.
__attribute__((visibility("default"))) size_t ref_observer_calls(size_t* out, size_t cap) {
  std::lock_guard<std::mutex> lock(g_obs_mu);
  for (size_t i = 0; i < g_obs.size() && i < cap; ++i) {
    out[2 * i] = g_obs[i].first;
    out[2 * i + 1] = g_obs[i].second;
  }
  return g_obs.size();
}

}  // extern "C"
