// tc16.cuh -- 256-point complex DFT on the tensor cores in split FP16: the
// precision variant of the multi-pass kernels' radix-16 stages.
//
// x[n1 * 16 + n2] (n1, n2 < 16) is a 16 x 16 matrix X; with F the 16-point
// DFT matrix (F[a][b] = w16^(ab)) and w256 the inter-stage twiddles,
//   Y = F X,  Y[k1][n2] *= w256^(k1 n2),  Z = Y F,  X_out[k1 + 16 k2] = Z[k1][k2].
// Each real product P Q of the complex GEMMs runs as P_hi Q_hi + P_hi Q_lo +
// P_lo Q_hi with P = P_hi + P_lo split into FP16 (the P_lo Q_lo term, about
// 2^-22 relative, is dropped), accumulated in FP32 by mma.sync m16n8k16.
// Before splitting, the block is scaled by a power of two so that its largest
// component lies in [0.5, 1) (per-block scaling: FP16's range is never
// exceeded and the split keeps 22 bits relative to the block maximum).  The
// stage-1 accumulators are laid out as the stage-2 A operand (rows g, g + 8,
// columns 2t, 2t + 1 (+8)), so the product never leaves registers.
//
// One warp transforms one 256-point block held in a padded shared-memory
// tile (pidx layout, natural order in and out).
#pragma once

#include <cuda_fp16.h>

#include "fft_engine.cuh"

namespace ffb {

__device__ __forceinline__ uint32_t pack_h2(float lo_col, float hi_col) {
  // low 16 bits: the lower column / row index of the pair
  const __half2 h = __floats2half2_rn(lo_col, hi_col);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// v = hi + lo in FP16 (hi rounded, lo the rounded remainder)
__device__ __forceinline__ void split2(float a, float b, uint32_t* hi, uint32_t* lo) {
  const __half2 h = __floats2half2_rn(a, b);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
  *hi = *reinterpret_cast<const uint32_t*>(&h);
  *lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += P Q in split FP16 (three products)
__device__ __forceinline__ void mma_split(float (&d)[4], const uint32_t (&ph)[4], const uint32_t (&pl)[4],
                                          uint32_t qh0, uint32_t qh1, uint32_t ql0, uint32_t ql1) {
  mma16816(d, ph, qh0, qh1);
  mma16816(d, ph, ql0, ql1);
  mma16816(d, pl, qh0, qh1);
}

// The warp's 256-point forward DFT of tile (pidx layout), in place.
__device__ __forceinline__ void tc_fft256(float2* tile, const Twiddles& tw) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // ---- constants: F as the stage-1 A operand (rows g, g+8; cols 2t, 2t+1, +8)
  //      and as the stage-2 B operand (rows 2t, 2t+1, +8; col g of tile j)
  uint32_t fa_rh[4], fa_rl[4], fa_ih[4], fa_il[4], fa_nih[4], fa_nil[4];
  {
    const int rows[4] = {g, g + 8, g, g + 8};
    const int cols[4] = {2 * t, 2 * t, 2 * t + 8, 2 * t + 8};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const float2 w0 = w16(rows[r] * cols[r]), w1 = w16(rows[r] * (cols[r] + 1));
      split2(w0.x, w1.x, &fa_rh[r], &fa_rl[r]);
      split2(w0.y, w1.y, &fa_ih[r], &fa_il[r]);
      split2(-w0.y, -w1.y, &fa_nih[r], &fa_nil[r]);
    }
  }
  uint32_t fb_rh[2][2], fb_rl[2][2], fb_ih[2][2], fb_il[2][2], fb_nih[2][2], fb_nil[2][2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int col = 8 * j + g;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int row = 2 * t + 8 * h;
      const float2 w0 = w16(row * col), w1 = w16((row + 1) * col);
      split2(w0.x, w1.x, &fb_rh[j][h], &fb_rl[j][h]);
      split2(w0.y, w1.y, &fb_ih[j][h], &fb_il[j][h]);
      split2(-w0.y, -w1.y, &fb_nih[j][h], &fb_nil[j][h]);
    }
  }
  // ---- X as the stage-1 B operand: tile j holds columns n2 = 8 j + g,
  //      rows n1 = 2t, 2t+1 (b0) and 2t+8, 2t+9 (b1)
  float2 x[2][4];
  float m = 0.f;
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int n1 = 2 * t + (e & 1) + 8 * (e >> 1);
      x[j][e] = tile[pidx(n1 * 16 + 8 * j + g)];
      m = fmaxf(m, fmaxf(fabsf(x[j][e].x), fabsf(x[j][e].y)));
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  int ex = 0;
  if (m > 0.f) (void)frexpf(m, &ex);  // m = f 2^ex, f in [0.5, 1)
  const float sc = ldexpf(1.f, -ex), inv = ldexpf(1.f, ex);
  // ---- stage 1: Y = F X
  float yr[2][4] = {}, yi[2][4] = {};
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    uint32_t xrh[2], xrl[2], xih[2], xil[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float2 p = x[j][2 * h], q = x[j][2 * h + 1];
      split2(p.x * sc, q.x * sc, &xrh[h], &xrl[h]);
      split2(p.y * sc, q.y * sc, &xih[h], &xil[h]);
    }
    // Yr = Fr Xr - Fi Xi, Yi = Fr Xi + Fi Xr
    mma_split(yr[j], fa_rh, fa_rl, xrh[0], xrh[1], xrl[0], xrl[1]);
    mma_split(yr[j], fa_nih, fa_nil, xih[0], xih[1], xil[0], xil[1]);
    mma_split(yi[j], fa_rh, fa_rl, xih[0], xih[1], xil[0], xil[1]);
    mma_split(yi[j], fa_ih, fa_il, xrh[0], xrh[1], xrl[0], xrl[1]);
  }
  // ---- inter-stage twiddles w256^(k1 n2): accumulator j, element e is
  //      row k1 = g (+8 for e >= 2), column n2 = 8 j + 2t + (e & 1)
  uint32_t ar_h[4], ar_l[4], ai_h[4], ai_l[4];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < 4; e += 2) {
      const int k1 = g + 4 * e;  // e = 0 -> g, e = 2 -> g + 8
      float2 y0 = make_float2(yr[j][e], yi[j][e]), y1 = make_float2(yr[j][e + 1], yi[j][e + 1]);
      const int n2 = 8 * j + 2 * t;
      y0 = cmul(y0, tw_get(tw, 8, (unsigned)(k1 * n2)));
      y1 = cmul(y1, tw_get(tw, 8, (unsigned)(k1 * (n2 + 1))));
      // A operand slot: a0 (row g, cols 2t..), a1 (row g+8), a2 (row g, cols +8), a3 (row g+8, cols +8)
      const int slot = (e >> 1) + 2 * j;
      split2(y0.x, y1.x, &ar_h[slot], &ar_l[slot]);
      split2(y0.y, y1.y, &ai_h[slot], &ai_l[slot]);
    }
  // ---- stage 2: Z = Y F; Zr = Yr Fr - Yi Fi, Zi = Yr Fi + Yi Fr
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    float zr[4] = {}, zi[4] = {};
    mma_split(zr, ar_h, ar_l, fb_rh[j][0], fb_rh[j][1], fb_rl[j][0], fb_rl[j][1]);
    mma_split(zr, ai_h, ai_l, fb_nih[j][0], fb_nih[j][1], fb_nil[j][0], fb_nil[j][1]);
    mma_split(zi, ar_h, ar_l, fb_ih[j][0], fb_ih[j][1], fb_il[j][0], fb_il[j][1]);
    mma_split(zi, ai_h, ai_l, fb_rh[j][0], fb_rh[j][1], fb_rl[j][0], fb_rl[j][1]);
    __syncwarp();  // every lane has read its inputs before the tile is overwritten
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k1 = g + 8 * (e >> 1), k2 = 8 * j + 2 * t + (e & 1);
      tile[pidx(k1 + 16 * k2)] = make_float2(zr[e] * inv, zi[e] * inv);
    }
  }
}

}  // namespace ffb
