// meta.cu -- metadata capture (reference eigen_fft.hpp:1477-1888, 3152-3168).
//
// The reference writes its metadata from inside its radix-2 executors.  Here
// the transform that carries metadata runs as that same literal radix-2
// stage sequence on the device, one launch per stage over every column:
//   Cooley-Tukey (eigen_fft.hpp:2655-3100): pre-hook, bit-reversal gather,
//     in-place stages len = 2..N, a = block*len + k, b = a + len/2,
//     w = W[k * N/len];
//   Stockham (eigen_fft.hpp:3227-3623): ping-pong stages s, seg = N>>(s+1),
//     in0 = 2j*seg + g, in1 = in0 + seg, out0 = j*seg + g, out1 = out0 + N/2,
//     w = W[j * seg];
// with the reference's own float twiddle table W (float angle arithmetic,
// computed on the host) and the butterfly t = b*w, (a + t, a - t) in
// round-to-nearest operations that the compiler may not contract, so the
// stage snapshots reproduce the reference's scalar arithmetic.  Integer
// metadata (layout, stage parameters, butterfly pairs, twiddle indices) is
// generated in closed form and is exact.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/fftfree_b200.h"
#include "context.h"
#include "kernels.h"

namespace ffb {

namespace {

__device__ __forceinline__ float2 bfly_mul(float2 b, float2 w) {
  return make_float2(__fsub_rn(__fmul_rn(b.x, w.x), __fmul_rn(b.y, w.y)),
                     __fadd_rn(__fmul_rn(b.x, w.y), __fmul_rn(b.y, w.x)));
}
__device__ __forceinline__ float norm2(float2 a) { return __fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)); }

// Non-negative floats order like their bit patterns as unsigned ints.
__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}

__device__ __forceinline__ void invariant(float* inv, int s, float2 a, float2 b, float2 y0, float2 y1) {
  // eigen_fft.hpp:2995-3003 / 3506-3523
  const float2 sum = make_float2(__fadd_rn(y0.x, y1.x), __fadd_rn(y0.y, y1.y));
  const float2 d = make_float2(__fsub_rn(sum.x, __fmul_rn(2.0f, a.x)), __fsub_rn(sum.y, __fmul_rn(2.0f, a.y)));
  const float r0 = hypotf(d.x, d.y);
  const float e = __fsub_rn(__fadd_rn(norm2(y0), norm2(y1)), __fmul_rn(2.0f, __fadd_rn(norm2(a), norm2(b))));
  atomic_max_pos(inv + 2 * s, r0);
  atomic_max_pos(inv + 2 * s + 1, fabsf(e));
}

__device__ __forceinline__ float2 pre_elem(const float2* col, int N, int n, int pre, int polar_in) {
  if (pre == 1) return make_float2(col[n].x, 0.f);
  if (pre == 2) {
    int m = n;
    bool cj = false;
    if (m > (N >> 1)) { m = N - m; cj = true; }
    float2 u = col[m];
    if (polar_in) {
      float s, c;
      sincosf(u.y, &s, &c);
      u = make_float2(u.x * c, u.x * s);
    }
    if (m == 0 || m == (N >> 1)) u.y = 0.f;
    return cj ? make_float2(u.x, -u.y) : u;
  }
  return col[n];
}

__device__ __forceinline__ int bitrev(int i, int lg) { return lg ? (int)(__brev((unsigned)i) >> (32 - lg)) : 0; }

__global__ void k_meta_load(const float2* in, float2* A, long long B, int N, int lg, int ct, int pre,
                            int polar_in) {
  const long long total = B * (long long)N;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long b = idx / N;
    const int i = (int)(idx - b * N);
    const int src = ct ? bitrev(i, lg) : i;
    A[idx] = pre_elem(in + b * N, N, src, ct ? pre : 0, polar_in);
  }
}

struct StageArgs {
  const float2* in;
  float2* out;  // == in for Cooley-Tukey
  const float2* W;
  long long B;
  int N, s;
  float2* snap;      // single snapshot (batch 0) or nullptr
  float2* snap_all;  // all batches or nullptr (Cooley-Tukey only)
  float* inv;        // 2 * S floats (r0, e) or nullptr
};

__global__ void k_ct_stage(StageArgs a) {
  const int half = 1 << a.s, len = half << 1, step = a.N / len;
  const long long per = a.N >> 1;
  const long long total = a.B * per;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long bb = idx / per;
    const int j = (int)(idx - bb * per);
    const int block = j / half, k = j - block * half;
    const int ia = block * len + k, ib = ia + half;
    float2* col = a.out + bb * a.N;
    const float2 va = col[ia], vb = col[ib];
    const float2 t = bfly_mul(vb, a.W[k * step]);
    const float2 y0 = make_float2(__fadd_rn(va.x, t.x), __fadd_rn(va.y, t.y));
    const float2 y1 = make_float2(__fsub_rn(va.x, t.x), __fsub_rn(va.y, t.y));
    col[ia] = y0;
    col[ib] = y1;
    if (a.snap_all) {
      float2* sa = a.snap_all + (long long)a.s * a.N * a.B + bb * a.N;
      sa[ia] = y0;
      sa[ib] = y1;
    } else if (a.snap && bb == 0) {
      a.snap[(long long)a.s * a.N + ia] = y0;
      a.snap[(long long)a.s * a.N + ib] = y1;
    }
    if (a.inv) invariant(a.inv, a.s, va, vb, y0, y1);
  }
}

__global__ void k_stockham_stage(StageArgs a) {
  const int seg = a.N >> (a.s + 1), halfN = a.N >> 1;
  const long long per = halfN;
  const long long total = a.B * per;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long bb = idx / per;
    const int u = (int)(idx - bb * per);
    const int j = u / seg, g = u - j * seg;
    const int i0 = 2 * j * seg + g, i1 = i0 + seg, o0 = j * seg + g, o1 = o0 + halfN;
    const float2* in = a.in + bb * a.N;
    float2* out = a.out + bb * a.N;
    const float2 va = in[i0], vb = in[i1];
    const float2 t = bfly_mul(vb, a.W[j * seg]);
    const float2 y0 = make_float2(__fadd_rn(va.x, t.x), __fadd_rn(va.y, t.y));
    const float2 y1 = make_float2(__fsub_rn(va.x, t.x), __fsub_rn(va.y, t.y));
    out[o0] = y0;
    out[o1] = y1;
    if (a.snap && bb == 0) {
      a.snap[(long long)a.s * a.N + o0] = y0;
      a.snap[(long long)a.s * a.N + o1] = y1;
    }
    if (a.inv) invariant(a.inv, a.s, va, vb, y0, y1);
  }
}

__global__ void k_meta_finish(const float2* A, float2* out, long long B, int N, int inverse, PostFlags pf) {
  const long long total = B * (long long)N;
  const float scale = 1.0f / (float)N;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(idx % N);
    float2 X = A[idx];
    if (inverse) X = make_float2(__fmul_rn(X.x, scale), __fmul_rn(X.y, scale));
    // post hook (eigen_fft.hpp:2535-2596)
    if (pf.r2c_half) {
      if (k > (N >> 1)) X = make_float2(0.f, 0.f);
      else if (k == 0 || k == (N >> 1)) X.y = 0.f;
    }
    if (pf.polar) X = make_float2(hypotf(X.x, X.y), atan2f(X.y, X.x));
    else if (pf.reduce) X = make_float2(hypotf(X.x, X.y), 0.f);
    else if (pf.clear_imag) X.y = 0.f;
    out[idx] = X;
  }
}

// Closed-form integer metadata: kind 4/9 ButterflyPairs(All), 6/10
// TwiddleIndexMap(All).  `reps` = batches for the All kinds (1 otherwise).
__global__ void k_meta_int(float2* buf, int kind, int N, int S, long long reps, int stockham) {
  const long long total = (long long)S * reps * N;
  const bool pairs = (kind == 4 || kind == 9);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long per = reps * N;
    const int s = (int)(idx / per);
    const int p = (int)(idx % N);
    float2 v;
    if (!stockham) {
      // eigen_fft.hpp:2953-3010
      const int half = 1 << s, len = half << 1;
      const int block = p / len, r = p - block * len;
      const int k = r & (half - 1);
      const int ia = block * len + k;
      v = pairs ? make_float2((float)ia, (float)(ia + half)) : make_float2((float)(k * (N / len)), 0.f);
    } else {
      // eigen_fft.hpp:3481-3505
      const int seg = N >> (s + 1), halfN = N >> 1;
      const int q = (p < halfN) ? p : p - halfN;
      const int j = q / seg, g = q - j * seg;
      const int i0 = 2 * j * seg + g;
      v = pairs ? make_float2((float)i0, (float)(i0 + seg)) : make_float2((float)(j * seg), 0.f);
    }
    buf[idx] = v;
  }
}

unsigned grid_for(long long total) {
  long long b = (total + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (unsigned)b;
}

bool dev_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

void ck(cudaError_t e) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "[fftfree_b200] CUDA error %s in metadata path: %s\n", cudaGetErrorName(e),
                 cudaGetErrorString(e));
    throw std::runtime_error("cuda");
  }
}

// Plan twiddle table of the reference (eigen_fft.hpp:2234-2242): float angle
// tau * k with tau = sgn * float(2 * acos(float(-1))) / float(N).
std::vector<float2> reference_twiddles(int N, bool inverse) {
  std::vector<float2> W(std::max(1, N / 2), make_float2(0.f, 0.f));
  const float sgn = inverse ? 1.0f : -1.0f;
  const float two_pi = 2 * std::acos(-1.0f);
  const float tau = sgn * two_pi / (float)N;
  for (int k = 0; k < N / 2; ++k) {
    const float ang = tau * (float)k;
    W[k] = make_float2(std::cos(ang), std::sin(ang));
  }
  return W;
}

struct Req {
  float2* user = nullptr;
  size_t count = 0;
  bool on_device = false;
};

}  // namespace

// Runs the metadata transform; returns 1, or 0 when a request is invalid.
int run_meta(FftContext* c, const float* in, float* out, size_t batch, const fftfree_metadata_request* reqs,
             int nreq) {
  const int N = c->N;
  int S = 0;
  while ((1 << S) < N) ++S;
  const size_t NS = (size_t)N * S;
  const bool stockham = c->stockham();
  const long long B = (long long)batch;
  // Writer construction and validation rules (eigen_fft.hpp:1529-1888).
  Req tw, lay, snap, params, pairs, inv, twmap, omega, snap_all, pairs_all, twmap_all;
  bool seen[11] = {false};
  for (int i = 0; i < nreq; ++i) {
    const int k = reqs[i].kind;
    float2* buf = reinterpret_cast<float2*>(reqs[i].buffer);
    const size_t cnt = reqs[i].count;
    if (k < 0 || k > 10) continue;
    if (k == 0) {
      size_t total = 0;
      for (int s = 0; s < S; ++s) total += (size_t)1 << s;
      if (total > 0 && (!buf || cnt < total)) return 0;
      tw.user = buf;
      tw.count = total;
      continue;
    }
    if (seen[k]) continue;
    seen[k] = true;
    auto need = [&](size_t n, Req& r, bool allow_null) -> bool {
      if (!buf) return allow_null;
      if (cnt < n) return false;
      r.user = buf;
      r.count = n;
      return true;
    };
    switch (k) {
      case 1: if (!need((size_t)N, lay, true)) return 0; break;
      case 2: if (S > 0 && !need(NS, snap, false)) return 0; break;
      case 3: if (S > 0 && !need((size_t)S, params, false)) return 0; break;
      case 4: if (S > 0 && !need(NS, pairs, false)) return 0; break;
      case 5: if (S > 0 && !need((size_t)S, inv, false)) return 0; break;
      case 6: if (S > 0 && !need(NS, twmap, false)) return 0; break;
      case 7: if (!stockham && !need((size_t)N, omega, true)) return 0; break;
      case 8: if (!stockham && S > 0 && !need(NS * batch, snap_all, false)) return 0; break;
      case 9: if (!stockham && S > 0 && !need(NS * batch, pairs_all, false)) return 0; break;
      case 10: if (!stockham && S > 0 && !need(NS * batch, twmap_all, false)) return 0; break;
    }
  }
  for (Req* r : {&tw, &lay, &snap, &params, &pairs, &inv, &twmap, &omega, &snap_all, &pairs_all, &twmap_all})
    if (r->user) r->on_device = dev_ptr(r->user);
  // CT quirk: the *All kinds take precedence over the single kinds
  // (eigen_fft.hpp:2981-3010), which are then left untouched.
  if (snap_all.user) snap.user = nullptr;
  if (pairs_all.user) pairs.user = nullptr;
  if (twmap_all.user) twmap.user = nullptr;

  cudaStream_t st = c->stream;
  auto put = [&](const Req& r, const std::vector<float2>& host) {
    if (!r.user || host.empty()) return;
    ck(cudaMemcpyAsync(r.user, host.data(), std::min(host.size(), r.count) * sizeof(float2),
                       r.on_device ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, st));
  };
  std::vector<float2> W = reference_twiddles(N, c->inverse);
  // host-side kinds
  std::vector<float2> h_tw, h_lay, h_params, h_omega;
  if (tw.user && tw.count) {
    h_tw.resize(tw.count);
    for (int s = 0; s < S; ++s) {
      const int m = 1 << s, step = N / (m << 1);
      for (int j = 0; j < m; ++j) h_tw[(m - 1) + j] = W[j * step];
    }
  }
  if (lay.user) {
    h_lay.resize(N);
    for (int p = 0; p < N; ++p) h_lay[p] = make_float2((float)p, 0.f);
  }
  if (params.user) {
    h_params.resize(S);
    for (int s = 0; s < S; ++s) h_params[s] = make_float2((float)(2 << s), (float)(N >> (s + 1)));
  }
  if (omega.user) {
    // OmegaMetadataWriter::fill (eigen_fft.hpp:1788-1798)
    const int upper = (c->eff_transform() == 1 && c->half_spectrum) ? N / 2 + 1 : N;
    const float two_pi = (float)(2 * std::acos(-1.0f));
    h_omega.resize(upper);
    for (int k = 0; k < upper; ++k) h_omega[k] = make_float2(two_pi * (float)k / (float)N, 0.f);
    omega.count = (size_t)upper;
  }

  // device work buffers
  const size_t n = (size_t)B * N;
  bool any_host = !dev_ptr(in) || !dev_ptr(out);
  const float2* d_in;
  if (dev_ptr(in)) {
    d_in = reinterpret_cast<const float2*>(in);
  } else {
    float2* t = static_cast<float2*>(c->d_in0.get(n * sizeof(float2)));
    ck(cudaMemcpyAsync(t, in, n * sizeof(float2), cudaMemcpyHostToDevice, st));
    d_in = t;
  }
  float2* A = static_cast<float2*>(c->d_frames.get(n * sizeof(float2)));
  float2* Bf = stockham ? static_cast<float2*>(c->d_out1.get(n * sizeof(float2))) : nullptr;
  float2* d_W = static_cast<float2*>(c->d_meta_tw.get(W.size() * sizeof(float2)));
  ck(cudaMemcpyAsync(d_W, W.data(), W.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  auto dev_target = [&](Req& r, DevBuf& tmp) -> float2* {
    if (!r.user) return nullptr;
    if (r.on_device) return r.user;
    return static_cast<float2*>(tmp.get(r.count * sizeof(float2)));
  };
  DevBuf t_snap, t_sall, t_inv, t_pairs, t_twmap;
  float2* d_snap = dev_target(snap, t_snap);
  float2* d_sall = dev_target(snap_all, t_sall);
  float* d_inv = nullptr;
  if (inv.user) {
    d_inv = static_cast<float*>(t_inv.get(2 * S * sizeof(float)));
    ck(cudaMemsetAsync(d_inv, 0, 2 * S * sizeof(float), st));
  }

  const int m = c->eff_transform();
  const int pre = (m == 1) ? 1 : ((m == 2 && c->half_spectrum) ? 2 : 0);
  k_meta_load<<<grid_for((long long)n), 256, 0, st>>>(d_in, A, B, N, S, stockham ? 0 : 1, pre,
                                                      c->store_polar ? 1 : 0);
  ++c->launches;
  float2* cur = A;
  float2* nxt = Bf;
  for (int s = 0; s < S; ++s) {
    StageArgs sa{};
    sa.W = d_W;
    sa.B = B;
    sa.N = N;
    sa.s = s;
    sa.snap = d_snap;
    sa.snap_all = stockham ? nullptr : d_sall;
    sa.inv = d_inv;
    const long long work = B * (N / 2);
    if (stockham) {
      sa.in = cur;
      sa.out = nxt;
      k_stockham_stage<<<grid_for(work), 256, 0, st>>>(sa);
      std::swap(cur, nxt);
    } else {
      sa.in = cur;
      sa.out = cur;
      k_ct_stage<<<grid_for(work), 256, 0, st>>>(sa);
    }
    ++c->launches;
  }
  // outputs
  float2* d_out;
  if (dev_ptr(out)) d_out = reinterpret_cast<float2*>(out);
  else d_out = static_cast<float2*>(c->d_out0.get(n * sizeof(float2)));
  k_meta_finish<<<grid_for((long long)n), 256, 0, st>>>(cur, d_out, B, N, c->inverse ? 1 : 0, c->post_flags());
  ++c->launches;
  ck(cudaGetLastError());
  if (!dev_ptr(out)) ck(cudaMemcpyAsync(out, d_out, n * sizeof(float2), cudaMemcpyDeviceToHost, st));

  auto int_kind = [&](Req& r, int kind, long long reps) {
    if (!r.user) return;
    DevBuf& tmp = (kind == 4 || kind == 9) ? t_pairs : t_twmap;
    float2* d = dev_target(r, tmp);
    const long long total = (long long)S * reps * N;
    k_meta_int<<<grid_for(total), 256, 0, st>>>(d, kind, N, S, reps, stockham ? 1 : 0);
    ++c->launches;
    ck(cudaGetLastError());
    if (!r.on_device) ck(cudaMemcpyAsync(r.user, d, r.count * sizeof(float2), cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));  // temp buffers are reused by the next kind
  };
  int_kind(pairs, 4, 1);
  int_kind(twmap, 6, 1);
  int_kind(pairs_all, 9, B);
  int_kind(twmap_all, 10, B);
  if (d_snap && !snap.on_device)
    ck(cudaMemcpyAsync(snap.user, d_snap, snap.count * sizeof(float2), cudaMemcpyDeviceToHost, st));
  if (d_sall && !snap_all.on_device)
    ck(cudaMemcpyAsync(snap_all.user, d_sall, snap_all.count * sizeof(float2), cudaMemcpyDeviceToHost, st));
  std::vector<float> h_inv;
  if (inv.user) {
    h_inv.resize(2 * S);
    ck(cudaMemcpyAsync(h_inv.data(), d_inv, 2 * S * sizeof(float), cudaMemcpyDeviceToHost, st));
  }
  ck(cudaStreamSynchronize(st));
  if (inv.user) {
    std::vector<float2> v(S);
    for (int s = 0; s < S; ++s) v[s] = make_float2(h_inv[2 * s], h_inv[2 * s + 1]);
    put(inv, v);
  }
  put(tw, h_tw);
  put(lay, h_lay);
  put(params, h_params);
  put(omega, h_omega);
  ck(cudaStreamSynchronize(st));
  (void)any_host;
  return 1;
}

}  // namespace ffb
