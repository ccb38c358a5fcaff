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

// Approximate reciprocal (PTX rcp.approx, documented to about one ulp; the
// parity tests bound its effect on the maps). The tensor-core epilogue's
// quotients use it: their divisors are
// bounded away from 0 and overflow (1 + t >= 1; the SSIM denominator >= c1 c2),
// and a correctly rounded reciprocal costs a multi-instruction sequence whose
// registers made the epilogue loop spill.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
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

// ---------------------------------------------------------------------------
// Packed FP32 pairs (sm_100 f32x2 arithmetic): two columns' terms per
// instruction. Used by the tensor-core engine's epilogue.
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

}  // namespace sred
