// Moment pass, relevance flags, compaction, operand packing and the per-pixel
// finalisation of the global repetition map.
//
// FP32 quantities that the reference computes (local statistics, noise tile
// variances, normalisation) are evaluated in the reference's own order with
// explicitly rounded operations (__fadd_rn etc., no FMA contraction) so that
// they agree bit for bit with an IEEE-754 evaluation of the reference code.
// Everything that feeds the all-pairs sums (block moments, unit vectors,
// weights' arguments, the per-pixel division) is FP64.
#include "common.cuh"
#include "kernels.cuh"

namespace sred {

int build_ellipse(int bw, int bh, Ellipse* e) {
  int rw = bw / 2, rh = bh / 2, k = 0;
  for (int y = -rh; y <= rh; y++)
    for (int x = -rw; x <= rw; x++) {
      float fx = (float)x, fy = (float)y;
      // java/GlobalRepetition2D_.java:107 (float arithmetic, same order)
      if (((fx * fx) / (float)(rw * rw)) + ((fy * fy) / (float)(rh * rh)) <= 1.0f) {
        if (k < kMaxK) {
          e->dx[k] = (short)x;
          e->dy[k] = (short)y;
        }
        k++;
      }
    }
  e->k = k;
  e->rw = rw;
  e->rh = rh;
  return k;
}

// ---------------------------------------------------------------------------
// Local statistics, cl/kernelGetLocalStatistics2D.cl:15-56 semantics.
// ---------------------------------------------------------------------------
__global__ void k_local_stats(const float* __restrict__ img, int W, int H, Ellipse e,
                              float* __restrict__ means, float* __restrict__ stds) {
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  int y = blockIdx.y;
  if (x >= W) return;
  size_t p = (size_t)y * W + x;
  if (x < e.rw || x >= W - e.rw || y < e.rh || y >= H - e.rh) {
    means[p] = 0.0f;
    stds[p] = 0.0f;
    return;
  }
  float s = 0.0f;
  for (int i = 0; i < e.k; i++) s = __fadd_rn(s, img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])]);
  float mean = __fdiv_rn(s, (float)e.k);
  float v = 0.0f;
  for (int i = 0; i < e.k; i++) {
    float d = __fsub_rn(img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])], mean);
    v = __fadd_rn(v, __fmul_rn(d, d));
  }
  v = __fdiv_rn(v, (float)(e.k - 1));
  means[p] = mean;
  stds[p] = __fsqrt_rn(v);
}

// ---------------------------------------------------------------------------
// Noise tiles, java/Utils.java:854-900: one thread per t x t tile, single
// pass over rows, FP32. bad != 0 if a NaN/Inf pixel is found in a tile.
// ---------------------------------------------------------------------------
__global__ void k_noise_tiles(const float* __restrict__ img, int W, int t, int nbx, int nb,
                              float* __restrict__ vars, int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  int bx = i % nbx, by = i / nbx;
  float mean = 0.0f, sq = 0.0f;
  int nonfinite = 0;
  for (int y = by * t; y < (by + 1) * t; y++)
    for (int x = bx * t; x < (bx + 1) * t; x++) {
      float v = img[(size_t)y * W + x];
      nonfinite |= !isfinite(v);
      mean = __fadd_rn(mean, v);
      sq = __fadd_rn(sq, __fmul_rn(v, v));
    }
  float n = (float)(t * t);
  mean = __fdiv_rn(mean, n);
  vars[i] = __fsub_rn(__fdiv_rn(sq, n), __fmul_rn(mean, mean));
  if (nonfinite) atomicOr(bad, 1);
}

// ---------------------------------------------------------------------------
// Relevance flags. mask: sigma^2 > threshold (java/Utils.java:957-965);
// relevant: !(sigma^2 < threshold) (cl/kernelGetGlobalPearson2D.cl:33,67);
// flat: sigma == 0 (cl/kernelGetGlobalPearson2D.cl:101-107).
// flags bit0 = relevant & !flat (gram list), bit1 = relevant & flat.
// If mask_in is given it is copied (the caller's RelevanceMask) instead of
// being derived, and n_mask counts mask > 0 on the interior.
// ---------------------------------------------------------------------------
__global__ void k_flags(const float* __restrict__ stds, const float* __restrict__ mask_in, int W, int H,
                        int rw, int rh, float thr, float* __restrict__ mask, uint8_t* __restrict__ flags,
                        unsigned long long* __restrict__ n_mask) {
  size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t n = (size_t)W * H;
  unsigned c = 0;
  if (p < n) {
    int x = (int)(p % W), y = (int)(p / W);
    bool interior = !(x < rw || x >= W - rw || y < rh || y >= H - rh);
    float s = stds[p];
    float s2 = __fmul_rn(s, s);
    float m;
    if (mask_in) m = mask_in[p];
    else m = (interior && !(s2 <= thr)) ? 1.0f : 0.0f;
    mask[p] = m;
    uint8_t f = 0;
    if (interior && !(s2 < thr)) f = (s == 0.0f) ? 2 : 1;
    flags[p] = f;
    c = (interior && m > 0.0f) ? 1u : 0u;
  }
  unsigned warp_c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && warp_c) atomicAdd(n_mask, (unsigned long long)warp_c);
}

// ---------------------------------------------------------------------------
// Deterministic stream compaction of the two flag classes (raster order).
// ---------------------------------------------------------------------------
constexpr int kSeg = kCompactSeg;  // pixels per compaction segment

__global__ void k_count(const uint8_t* __restrict__ flags, size_t n, int2* __restrict__ counts) {
  size_t base = (size_t)blockIdx.x * kSeg;
  int a = 0, b = 0;
  for (int i = threadIdx.x; i < kSeg; i += blockDim.x) {
    size_t p = base + i;
    if (p < n) {
      uint8_t f = flags[p];
      a += (f == 1);
      b += (f == 2);
    }
  }
  a = __reduce_add_sync(0xffffffffu, a);
  b = __reduce_add_sync(0xffffffffu, b);
  __shared__ int sa[32], sb[32];
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    int ta = 0, tb = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) { ta += sa[i]; tb += sb[i]; }
    counts[blockIdx.x] = make_int2(ta, tb);
  }
}

// Single-CTA exclusive scan over segment counts; totals written at [nseg].
__global__ void k_scan(int2* __restrict__ counts, int nseg) {
  __shared__ int2 carry;
  if (threadIdx.x == 0) carry = make_int2(0, 0);
  __syncthreads();
  for (int base = 0; base < nseg; base += blockDim.x) {
    int i = base + threadIdx.x;
    int2 v = i < nseg ? counts[i] : make_int2(0, 0);
    // inclusive warp scan
    int a = v.x, b = v.y;
    for (int o = 1; o < 32; o <<= 1) {
      int ta = __shfl_up_sync(0xffffffffu, a, o), tb = __shfl_up_sync(0xffffffffu, b, o);
      if ((threadIdx.x & 31) >= o) { a += ta; b += tb; }
    }
    __shared__ int2 wsum[32];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 31) wsum[w] = make_int2(a, b);
    __syncthreads();
    if (w == 0) {
      int nw = blockDim.x >> 5;
      int2 s = l < nw ? wsum[l] : make_int2(0, 0);
      int sa = s.x, sb = s.y;
      for (int o = 1; o < 32; o <<= 1) {
        int ta = __shfl_up_sync(0xffffffffu, sa, o), tb = __shfl_up_sync(0xffffffffu, sb, o);
        if (l >= o) { sa += ta; sb += tb; }
      }
      if (l < nw) wsum[l] = make_int2(sa - s.x, sb - s.y);  // exclusive warp offsets
    }
    __syncthreads();
    int2 c = carry;
    int ea = a - v.x + wsum[w].x + c.x, eb = b - v.y + wsum[w].y + c.y;
    if (i < nseg) counts[i] = make_int2(ea, eb);
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = make_int2(ea + v.x, eb + v.y);
    __syncthreads();
  }
  if (threadIdx.x == 0) counts[nseg] = carry;
}

// slot[p] = gram index (>= 0), -(flat index) - 2 for flat, -1 otherwise.
__global__ void k_scatter(const uint8_t* __restrict__ flags, size_t n, const int2* __restrict__ offs,
                          int* __restrict__ gram_pix, int* __restrict__ flat_pix, int* __restrict__ slot) {
  size_t base = (size_t)blockIdx.x * kSeg;
  int2 o = offs[blockIdx.x];
  __shared__ int2 wtot[8];
  __shared__ int2 run;
  if (threadIdx.x == 0) run = o;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int c0 = 0; c0 < kSeg; c0 += blockDim.x) {
    size_t p = base + c0 + threadIdx.x;
    uint8_t f = p < n ? flags[p] : 0;
    unsigned ba = __ballot_sync(0xffffffffu, f == 1), bb = __ballot_sync(0xffffffffu, f == 2);
    if (lane == 0) wtot[w] = make_int2(__popc(ba), __popc(bb));
    __syncthreads();
    int pa = run.x, pb = run.y;
    for (int i = 0; i < w; i++) { pa += wtot[i].x; pb += wtot[i].y; }
    unsigned lt = (1u << lane) - 1u;
    if (p < n) {
      if (f == 1) {
        int j = pa + __popc(ba & lt);
        gram_pix[j] = (int)p;
        slot[p] = j;
      } else if (f == 2) {
        int j = pb + __popc(bb & lt);
        flat_pix[j] = (int)p;
        slot[p] = -j - 2;
      } else {
        slot[p] = -1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int ta = 0, tb = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) { ta += wtot[i].x; tb += wtot[i].y; }
      run = make_int2(run.x + ta, run.y + tb);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Operand packing: each warp takes 32 consecutive gram blocks at a time (their
// pixels overlap, so the passes hit L1). FP64 moments of the ellipse vector,
// unit vector u = (x - mu) / |x - mu|, per-block epilogue params, and the
// closed-form sums the flat blocks need:
//   sums[0] = sum_q 2^-(a_q)^2           (weight of a pair with a flat block)
//   sums[1] = sum_q sqrt((K-1)/K) sigma_q (NRMSE against a flat block)
//   sums[2] = sum_q sigma_q 2^-(a_q)^2     (Abs-diff against a flat block)
// The block sums are warp-wide reductions, one block after another; the
// per-block scalar work (square roots, quotients, exp2, params) then runs on
// lane k for block k of the 32, instead of on one lane per block while the
// other 31 wait. mode 0: U only (fp32, row pitch kp). mode 1 / 2: the two- /
// three-level split BF16 operands A, B (store_split; row pitch kq), and U as
// well when U is given (tensor-core NRMSE). Rows [n, n_pad) are zero-filled by
// the host.
// ---------------------------------------------------------------------------
__global__ void k_pack(const float* __restrict__ img, int W, Ellipse e, const int* __restrict__ gram_pix,
                       int n, float wscale, int mode, float* __restrict__ U, int kp,
                       __nv_bfloat16* __restrict__ A, __nv_bfloat16* __restrict__ B, int kq,
                       BlockParams* __restrict__ params, float* __restrict__ tile_rmax,
                       double* __restrict__ sums) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int K = e.k;
  const double sk = sqrt((double)(K - 1) / (double)K);
  const double rK = __drcp_rn((double)K);  // s / K as div_fixed: the correctly rounded quotient
  double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
  for (long long j0 = 32LL * gw; j0 < n; j0 += 32LL * nw) {
    const int nb = (int)min(32LL, (long long)n - j0);
    // The sum and centred sum of squares of each block; lane k keeps block k's.
    double my_s = 0.0, my_v = 0.0;
    for (int k = 0; k < nb; k++) {
      const int p = gram_pix[j0 + k];
      const int x = p % W, y = p / W;
      double s = 0.0;
      for (int i = lane; i < K; i += 32) s += (double)img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])];
      for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(full, s, o);
      const double mu = div_fixed(s, (double)K, rK);
      double v = 0.0;
      for (int i = lane; i < K; i += 32) {
        const double d = (double)img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])] - mu;
        v += d * d;
      }
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(full, v, o);
      if (lane == k) {
        my_s = s;
        my_v = v;
      }
    }
    // Block j0 + lane's scalars.
    double mu = 0.0, inv = 0.0;
    if (lane < nb) {
      const long long j = j0 + lane;
      mu = div_fixed(my_s, (double)K, rK);
      const double nrm = sqrt(my_v);
      inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
      const double sigma = sqrt(my_v / (K - 1));
      BlockParams bp;
      bp.a = (float)(sigma * (double)wscale);
      bp.e = sigma > 0.0 ? (float)((double)kEps / sigma) : 0.0f;
      bp.r = sigma > 0.0 ? (float)(1.0 / sigma) : 0.0f;
      bp.sigma = (float)sigma;
      bp.mu = (float)mu;
      bp.pad0 = bp.pad1 = bp.pad2 = 0.0f;
      params[j] = bp;
      atomicMax(reinterpret_cast<int*>(tile_rmax) + (j >> 7), __float_as_int(bp.r));
      const double a = sigma * (double)wscale;
      const double w0 = exp2(-(a * a));
      acc0 += w0;
      acc1 += sk * sigma;
      acc2 += sigma * w0;
    }
    // Unit vectors and operands, block by block.
    for (int k = 0; k < nb; k++) {
      const long long j = j0 + k;
      const double mu_k = __shfl_sync(full, mu, k), inv_k = __shfl_sync(full, inv, k);
      const int p = gram_pix[j];
      const int x = p % W, y = p / W;
      for (int i = lane; i < K; i += 32) {
        const double u = ((double)img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])] - mu_k) * inv_k;
        if (U) U[(size_t)j * kp + i] = (float)u;
        if (mode != 0) store_split(A + (size_t)j * kq, B + (size_t)j * kq, K, i, u, mode + 1);
      }
      if (U)
        for (int i = K + lane; i < kp; i += 32) U[(size_t)j * kp + i] = 0.0f;
      if (mode != 0) {
        for (int i = (mode == 1 ? 3 : 6) * K + lane; i < kq; i += 32) {
          A[(size_t)j * kq + i] = __float2bfloat16_rn(0.0f);
          B[(size_t)j * kq + i] = __float2bfloat16_rn(0.0f);
        }
      }
    }
  }
  for (int o = 16; o; o >>= 1) {
    acc0 += __shfl_xor_sync(full, acc0, o);
    acc1 += __shfl_xor_sync(full, acc1, o);
    acc2 += __shfl_xor_sync(full, acc2, o);
  }
  __shared__ double red[3][32];
  const int wi = threadIdx.x >> 5;
  if (lane == 0) { red[0][wi] = acc0; red[1][wi] = acc1; red[2][wi] = acc2; }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += red[threadIdx.x][i];
    atomicAdd(sums + threadIdx.x, t);
  }
}

// Diagnostics: pack caller-given vectors (n x K, FP32) as operands without
// normalising them (one warp per row).
__global__ void k_pack_vectors(const float* __restrict__ u, int n, int K, int mode, float* __restrict__ U, int kp,
                               __nv_bfloat16* __restrict__ A, __nv_bfloat16* __restrict__ B, int kq) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int j = gw; j < n; j += nw) {
    if (mode == 0) {
      for (int i = lane; i < kp; i += 32) U[(size_t)j * kp + i] = i < K ? u[(size_t)j * K + i] : 0.0f;
    } else {
      for (int i = lane; i < kq; i += 32) {
        A[(size_t)j * kq + i] = __float2bfloat16_rn(0.0f);
        B[(size_t)j * kq + i] = __float2bfloat16_rn(0.0f);
      }
      __syncwarp();
      for (int i = lane; i < K; i += 32) {
        const float x = u[(size_t)j * K + i];
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
        __nv_bfloat16* a = A + (size_t)j * kq;
        __nv_bfloat16* b = B + (size_t)j * kq;
        a[i] = hi; a[K + i] = lo; a[2 * K + i] = hi;
        b[i] = hi; b[K + i] = hi; b[2 * K + i] = lo;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Finalisation, java/CLUtils.java:1747-1770, :1998-2027, :2127-2156:
// out = num / (den * nPixels + eps) (FP64 here), the NRMSE / Abs-diff
// inversion on mask > 0, and the mask when the relevance constant is > 0.
// The closed-form flat-block contributions are added here.
// ---------------------------------------------------------------------------
__global__ void k_finalize(const int* __restrict__ slot, int W, int H, int rw, int rh,
                           const double* __restrict__ num, const double* __restrict__ den,
                           const BlockParams* __restrict__ params, const double* __restrict__ sums,
                           int n_flat, int metric, double sk, double n_pixels, const float* __restrict__ mask,
                           int apply_mask, float* __restrict__ out) {
  size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (size_t)W * H) return;
  int x = (int)(p % W), y = (int)(p / W);
  float o = 0.0f;
  if (!(x < rw || x >= W - rw || y < rh || y >= H - rh)) {
    int s = slot[p];
    double nu = 0.0, de = 0.0;
    if (s >= 0) {
      BlockParams bp = params[s];
      double a = (double)bp.a;
      double w0 = exp2(-(a * a));
      nu = num[s];
      de = den[s] + (double)n_flat * w0;
      if (metric == kNrmse) nu += (double)n_flat * sk * (double)bp.sigma;
      else if (metric == kAbsDiff) nu += (double)n_flat * (double)bp.sigma * w0;
    } else if (s <= -2) {
      de = sums[0] + (double)n_flat;
      if (metric == kPearson || metric == kSsim) nu = (double)n_flat;
      else if (metric == kNrmse) nu = sums[1];
      else nu = sums[2];
    }
    o = (float)(nu / (de * n_pixels + (double)kEps));
    // Inversion of the FP32 value, as java/CLUtils.java:1998-2010 does it
    // (a value that rounds to 0 becomes 1, a denormal becomes inf).
    if ((metric == kNrmse || metric == kAbsDiff) && mask[p] > 0.0f) o = (o == 0.0f) ? 1.0f : __fdiv_rn(1.0f, o);
    if (apply_mask) o = __fmul_rn(o, mask[p]);
  }
  out[p] = o;
}

// ---------------------------------------------------------------------------
// Normalisation, java/Utils.java:985-1031: min/max over mask > 0 on the
// interior (or the whole interior when mask is NULL), then
// (v - min) / (max - min + eps) in FP32.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ord_bits(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_float(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_minmax(const float* __restrict__ a, const float* __restrict__ mask, int W, int H,
                         int bw_, int bh_, size_t plane, unsigned* __restrict__ mm) {
  const float* img = a + plane * blockIdx.y;
  const float* msk = mask ? mask + plane * blockIdx.y : nullptr;
  unsigned* m = mm + 2 * blockIdx.y;
  unsigned lo = 0xffffffffu, hi = 0u;
  size_t n = (size_t)W * H;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int x = (int)(p % W), y = (int)(p / W);
    if (x < bw_ || x >= W - bw_ || y < bh_ || y >= H - bh_) continue;
    if (msk && !(msk[p] > 0.0f)) continue;
    unsigned b = ord_bits(img[p]);
    lo = min(lo, b);
    hi = max(hi, b);
  }
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(m, lo);
    atomicMax(m + 1, hi);
  }
}

__global__ void k_remap(float* __restrict__ a, const float* __restrict__ mask, int W, int H, int bw_,
                        int bh_, size_t plane, const unsigned* __restrict__ mm) {
  float* img = a + plane * blockIdx.y;
  const float* msk = mask ? mask + plane * blockIdx.y : nullptr;
  const unsigned* m = mm + 2 * blockIdx.y;
  if (m[1] == 0u) return;  // nothing selected: the reference remaps nothing either
  float mn = ord_float(m[0]), mx = ord_float(m[1]);
  float d = __fadd_rn(__fsub_rn(mx, mn), kEps);
  size_t n = (size_t)W * H;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    int x = (int)(p % W), y = (int)(p / W);
    if (x < bw_ || x >= W - bw_ || y < bh_ || y >= H - bh_) continue;
    if (msk && !(msk[p] > 0.0f)) continue;
    img[p] = __fdiv_rn(__fsub_rn(img[p], mn), d);
  }
}

}  // namespace sred
