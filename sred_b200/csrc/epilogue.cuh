// Fused per-pair epilogue of the global repetition map, shared by the FP32
// CUDA-core engine and the split-BF16 tensor-core engine.
//
// Input per pair (p, q): G = <u_p, u_q>, the dot product of the two blocks'
// zero-mean unit vectors (the contraction engine's output), and the blocks'
// FP64-derived parameters. The reference's per-pair quantities
// (cl/kernelGetGlobal*2D.cl) are rewritten in terms of G:
//   cov_pq            = sigma_p sigma_q G                  (K-1 normalisation)
//   weight            = exp(-(sigma_p - sigma_q)^2 / (v + eps)) = 2^-(a_p - a_q)^2
//   Pearson           = max(0, G sigma_p sigma_q / (sigma_p sigma_q + eps)) * weight
//                     = max(0, G / (1 + t)) * weight,  t = (eps / sigma_p)(1 / sigma_q)
//   SSIM (global)     = max(0, (2 mu_p mu_q + c1)(2 cov + c2) /
//                              ((mu_p^2 mu_q^2 + c1)(sigma_p^2 + sigma_q^2 + c2)) * weight)
//   NRMSE (unweighted)= sqrt(((K-1)/K) ((sigma_p - sigma_q)^2 + 2 sigma_p sigma_q (1 - G)))
//   Abs-diff          = |sigma_p - sigma_q| * weight
// The NRMSE form uses the normalised vectors, so the large common part of
// |x_p|^2 + |x_q|^2 - 2<x_p, x_q> never cancels in FP32.
// 1/(1+t) is evaluated to first or second order, or exactly, according to the
// tile's largest t (c_mode below), with relative error below 6e-8.
// The self pair (q == p) uses G = 1 exactly, as the reference's direct
// evaluation gives; only tiles that contain the diagonal check for it.
#pragma once
#include "common.cuh"

namespace sred {

constexpr float kTFast = 1.0f / 256.0f;

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct RowState {
  float a, e, r, sigma, mu;
  float mu2x2;   // 2 mu_p
  float mumu;    // mu_p^2
  float s2;      // sigma_p^2 + c2
  float sig2x;   // 2 sigma_p
};

__device__ __forceinline__ RowState make_row(const BlockParams& bp, const EpiConsts& ec) {
  RowState r;
  r.a = bp.a;
  r.e = bp.e;
  r.r = bp.r;
  r.sigma = bp.sigma;
  r.mu = bp.mu;
  r.mu2x2 = 2.0f * bp.mu;
  r.mumu = bp.mu * bp.mu;
  r.s2 = bp.sigma * bp.sigma + ec.c2;
  r.sig2x = 2.0f * bp.sigma;
  return r;
}

// Evaluation of the Pearson factor 1/(1+t), chosen per tile from the tile's
// largest t = eps / (sigma_p sigma_q):
//   kCFirst  t < 2^-13: G (1 - t)          (relative error t^2 < 1.5e-8)
//   kCSecond t < 2^-8:  G (1 - t + t^2)    (relative error t^3 < 6e-8)
//   kCExact  otherwise: G / (1 + t)
enum { kCFirst = 0, kCSecond = 1, kCExact = 2 };
constexpr float kTFirst = 1.0f / 8192.0f;

__device__ __forceinline__ int c_mode(float tmax) {
  return tmax < kTFirst ? kCFirst : (tmax < kTFast ? kCSecond : kCExact);
}

// The two per-pair terms (numerator tn, denominator td); symmetric in p, q.
// CMODE is used by Pearson only.
template <int METRIC, int CMODE>
__device__ __forceinline__ void pair_terms(float G, const RowState& rp, const BlockParams& cq,
                                           const EpiConsts& ec, float& tn, float& td) {
  if (METRIC == kDebugDot) {  // symmetric diagnostic terms
    tn = G * rp.a * cq.a;
    td = rp.r + cq.r;
    return;
  }
  const float d = rp.a - cq.a;
  const float w = ex2_approx(-d * d);
  td = w;
  if (METRIC == kPearson) {
    float gc;
    if (CMODE == kCFirst) {
      gc = fmaf(-G * rp.e, cq.r, G);
    } else if (CMODE == kCSecond) {
      const float t = rp.e * cq.r;
      gc = G * fmaf(t, t - 1.0f, 1.0f);
    } else {
      gc = G * __frcp_rn(1.0f + rp.e * cq.r);
    }
    tn = fmaxf(gc, 0.0f) * w;
  } else if (METRIC == kSsim) {
    const float num = fmaf(rp.mu2x2, cq.mu, ec.c1) * fmaf(rp.sig2x * cq.sigma, G, ec.c2);
    const float den = fmaf(rp.mumu, cq.mu * cq.mu, ec.c1) * fmaf(cq.sigma, cq.sigma, rp.s2);
    tn = fmaxf(__fdividef(num, den) * w, 0.0f);
  } else if (METRIC == kNrmse || METRIC == kNrmseW) {
    const float ds = rp.sigma - cq.sigma;
    const float m = ec.nrmse_scale * fmaf(ds, ds, rp.sig2x * cq.sigma * (1.0f - G));
    tn = sqrtf(fmaxf(m, 0.0f));
    if (METRIC == kNrmseW) tn *= w;
  } else if (METRIC == kNrmseD || METRIC == kNrmseDW) {
    // G holds |u_p - u_q|^2 = 2 (1 - <u_p, u_q>): both terms are >= 0, so
    // near-identical blocks lose nothing to cancellation.
    const float ds = rp.sigma - cq.sigma;
    tn = sqrtf(ec.nrmse_scale * fmaf(ds, ds, rp.sigma * cq.sigma * G));
    if (METRIC == kNrmseDW) tn *= w;
  } else {  // Abs-diff of stds
    tn = fabsf(rp.sigma - cq.sigma) * w;
  }
}

// One pair accumulated into the row sums.
template <int METRIC, int CMODE>
__device__ __forceinline__ void epi_pair(float G, const RowState& rp, const BlockParams& cq,
                                         const EpiConsts& ec, float& sn, float& sd) {
  float tn, td;
  pair_terms<METRIC, CMODE>(G, rp, cq, ec, tn, td);
  sn += tn;
  sd += td;
}

// ---------------------------------------------------------------------------
// Packed FP32 pairs (sm_100 f32x2 arithmetic): two columns' terms per
// instruction. Used by the tensor-core engine's Pearson fast path.
// ---------------------------------------------------------------------------
struct F2 {
  unsigned long long v;
};

__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_split(F2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 sub2(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {  // a * b + c
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// Row constants of the packed Pearson path, both halves equal.
struct PearsonRow2 {
  F2 a, e, ne, m1, one;
};

__device__ __forceinline__ PearsonRow2 make_pearson_row2(const RowState& rs) {
  PearsonRow2 r;
  r.a = f2(rs.a, rs.a);
  r.e = f2(rs.e, rs.e);
  r.ne = f2(-rs.e, -rs.e);
  r.m1 = f2(-1.0f, -1.0f);
  r.one = f2(1.0f, 1.0f);
  return r;
}

// Two Pearson pairs (columns q0, q1 of one row), the terms of pair_terms for
// CMODE kCFirst / kCSecond, accumulated into packed sums (numerator with one
// fused multiply-add).
template <int CMODE>
__device__ __forceinline__ void pearson_pair2(F2 G, F2 aq, F2 rq, const PearsonRow2& r, F2& sn, F2& sd) {
  const F2 d = sub2(r.a, aq);
  float m0, m1;
  f2_split(mul2(d, d), m0, m1);
  const F2 w = f2(ex2_approx(-m0), ex2_approx(-m1));
  F2 gc;
  if (CMODE == kCFirst) {
    gc = fma2(mul2(G, r.ne), rq, G);  // G - G e_p r_q
  } else {
    const F2 t = mul2(r.e, rq);
    gc = mul2(G, fma2(t, add2(t, r.m1), r.one));  // G (1 - t + t^2)
  }
  float g0, g1;
  f2_split(gc, g0, g1);
  sn = fma2(f2(fmaxf(g0, 0.0f), fmaxf(g1, 0.0f)), w, sn);
  sd = add2(sd, w);
}

// Row constants of the packed SSIM path, both halves equal.
struct SsimRow2 {
  F2 a, mu2x2, sig2x, mumu, s2, c1, c2;
};

__device__ __forceinline__ SsimRow2 make_ssim_row2(const RowState& rs, const EpiConsts& ec) {
  SsimRow2 r;
  r.a = f2(rs.a, rs.a);
  r.mu2x2 = f2(rs.mu2x2, rs.mu2x2);
  r.sig2x = f2(rs.sig2x, rs.sig2x);
  r.mumu = f2(rs.mumu, rs.mumu);
  r.s2 = f2(rs.s2, rs.s2);
  r.c1 = f2(ec.c1, ec.c1);
  r.c2 = f2(ec.c2, ec.c2);
  return r;
}

// Two SSIM pairs (columns q0, q1 of one row): pair_terms' kSsim arithmetic,
// operation for operation, on f32x2 pairs (the quotient and the weight per
// half), accumulated into packed sums.
__device__ __forceinline__ void ssim_pair2(F2 G, F2 aq, F2 sq, F2 mq, const SsimRow2& r, F2& sn, F2& sd) {
  const F2 d = sub2(r.a, aq);
  float m0, m1;
  f2_split(mul2(d, d), m0, m1);
  const F2 w = f2(ex2_approx(-m0), ex2_approx(-m1));
  const F2 num = mul2(fma2(r.mu2x2, mq, r.c1), fma2(mul2(r.sig2x, sq), G, r.c2));
  const F2 den = mul2(fma2(r.mumu, mul2(mq, mq), r.c1), fma2(sq, sq, r.s2));
  float n0, n1, d0, d1;
  f2_split(num, n0, n1);
  f2_split(den, d0, d1);
  float t0, t1;
  f2_split(mul2(f2(__fdividef(n0, d0), __fdividef(n1, d1)), w), t0, t1);
  sn = add2(sn, f2(fmaxf(t0, 0.0f), fmaxf(t1, 0.0f)));
  sd = add2(sd, w);
}

// Column sums of 16 columns over the 32 lanes of a warp (lane l holds row l's
// terms x[0..15]): four butterfly exchanges halve the columns each lane keeps,
// a fifth adds the lane pairs. Afterwards lanes 2c and 2c+1 both hold the sum
// of column c over all 32 rows.
__device__ __forceinline__ float lane_column_sums16(const float (&x)[16]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float y8[8], y4[4], y2[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4, b1 = lane & 2;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const float send = b4 ? x[i] : x[i + 8], keep = b4 ? x[i + 8] : x[i];
    y8[i] = keep + __shfl_xor_sync(full, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float send = b3 ? y8[i] : y8[i + 4], keep = b3 ? y8[i + 4] : y8[i];
    y4[i] = keep + __shfl_xor_sync(full, send, 8);
  }
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const float send = b2 ? y4[i] : y4[i + 2], keep = b2 ? y4[i + 2] : y4[i];
    y2[i] = keep + __shfl_xor_sync(full, send, 4);
  }
  const float send = b1 ? y2[0] : y2[1], keep = b1 ? y2[1] : y2[0];
  float y = keep + __shfl_xor_sync(full, send, 2);
  return y + __shfl_xor_sync(full, y, 1);
}

}  // namespace sred
