// Variance stabilisation by the quadtree / octree method ("Quad/Octree",
// java/QuadTree_.java and java/OcTree_.java): per-node statistics of the
// tree's Fisher-test split criterion, and per-leaf robust means and
// least-trimmed-squares variances, one CTA per node or leaf. The tree itself,
// the F quantiles and the regression are host code (sred_api.cu).
//
// Sums are FP64 in a fixed order (a strided thread loop, then a pairwise tree
// over the CTA); the reference sums in FP32 in raster order, so values agree
// to FP32 rounding, not bit for bit.
#include "gat_tree.cuh"

namespace sred {

namespace {

constexpr int kT = kTreeThreads;

__device__ __forceinline__ double cta_sum(double v, double* s) {
  s[threadIdx.x] = v;
  __syncthreads();
  for (int st = kT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
    __syncthreads();
  }
  const double r = s[0];
  __syncthreads();
  return r;
}

// Voxel i (raster order z, y, x) of a box.
__device__ __forceinline__ size_t box_index(const TreeBox& b, size_t i, int W, int H) {
  const size_t bw = b.w, bh = b.h;
  const size_t x = b.x + i % bw, y = b.y + (i / bw) % bh, z = b.z + i / (bw * bh);
  return (z * H + y) * W + x;
}

// Pseudo-residual of one voxel: (l v - the neighbours inside the image) *
// 1/sqrt(l^2 + l), FP32 in the reference's order (l = 5 with 4 neighbours in
// 2D, 7 with 6 in 3D).
__device__ __forceinline__ float pseudo_residual(const float* img, int W, int H, int D, size_t p, int x, int y,
                                                 int z, bool three_d, float scale) {
  const float l = three_d ? 7.0f : 5.0f;
  float lap = l * img[p];
  if (x > 0) lap -= img[p - 1];
  if (x < W - 1) lap -= img[p + 1];
  if (y > 0) lap -= img[p - W];
  if (y < H - 1) lap -= img[p + W];
  if (three_d) {
    if (z > 0) lap -= img[p - (size_t)W * H];
    if (z < D - 1) lap -= img[p + (size_t)W * H];
  }
  return lap * scale;
}

}  // namespace

// Per node: out[2 i] = block variance (sum v^2 / n - mean^2), out[2 i + 1] =
// variance of the pseudo-residuals (two passes, divided by n - 1).
__global__ void __launch_bounds__(kTreeThreads)
    k_tree_node_stats(const float* __restrict__ img, int W, int H, int D, const TreeBox* __restrict__ boxes,
                      int three_d, float scale, double* __restrict__ out) {
  __shared__ double s[kT];
  const TreeBox b = boxes[blockIdx.x];
  const size_t n = (size_t)b.w * b.h * b.d;
  double s1 = 0.0, s2 = 0.0, r1 = 0.0;
  for (size_t i = threadIdx.x; i < n; i += kT) {
    const size_t p = box_index(b, i, W, H);
    const int x = (int)(p % W), y = (int)((p / W) % H), z = (int)(p / ((size_t)W * H));
    const double v = (double)img[p];
    s1 += v;
    s2 += v * v;
    r1 += (double)pseudo_residual(img, W, H, D, p, x, y, z, three_d, scale);
  }
  s1 = cta_sum(s1, s);
  s2 = cta_sum(s2, s);
  r1 = cta_sum(r1, s);
  const double mr = r1 / (double)n;
  double r2 = 0.0;
  for (size_t i = threadIdx.x; i < n; i += kT) {
    const size_t p = box_index(b, i, W, H);
    const int x = (int)(p % W), y = (int)((p / W) % H), z = (int)(p / ((size_t)W * H));
    const double d = (double)pseudo_residual(img, W, H, D, p, x, y, z, three_d, scale) - mr;
    r2 += d * d;
  }
  r2 = cta_sum(r2, s);
  if (threadIdx.x == 0) {
    const double m = s1 / (double)n;
    out[2 * blockIdx.x] = s2 / (double)n - m * m;
    out[2 * blockIdx.x + 1] = r2 / ((double)n - 1.0);
  }
}

// Robust mean of each leaf (QuadTree_.calculateRobustMean): the starting
// variance is the reference's running-sum expression sum_i (v_i - S_i)^2 /
// (n - 1) with S_i the running sum (= sum_i S_{i-1}^2 / (n - 1)), at least
// eps; then Gaussian-weighted means until the mean moves by at most 1e-5 or
// max_iter rounds. The running sum is a CTA scan over the leaf in raster
// order, FP64.
__global__ void __launch_bounds__(kTreeThreads)
    k_tree_robust_mean(const float* __restrict__ img, int W, int H, const TreeBox* __restrict__ boxes,
                       int max_iter, float* __restrict__ out) {
  __shared__ double s[kT];
  __shared__ double carry;
  const TreeBox b = boxes[blockIdx.x];
  const size_t n = (size_t)b.w * b.h * b.d;
  if (threadIdx.x == 0) carry = 0.0;
  __syncthreads();
  double q = 0.0;
  for (size_t base = 0; base < n; base += kT) {
    const size_t i = base + threadIdx.x;
    const double v = i < n ? (double)img[box_index(b, i, W, H)] : 0.0;
    // inclusive scan of v over the chunk (Hillis-Steele in shared memory)
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < kT; o <<= 1) {
      const double t = threadIdx.x >= o ? s[threadIdx.x - o] : 0.0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    const double excl = carry + s[threadIdx.x] - v;  // S_{i-1}
    if (i < n) q += excl * excl;
    __syncthreads();
    if (threadIdx.x == kT - 1) carry += s[kT - 1];
    __syncthreads();
  }
  const double total = carry;
  q = cta_sum(q, s);
  float mean = (float)(total / (double)n);
  const float var = fmaxf((float)(q / ((double)n - 1.0)), kEps);
  __shared__ float smean;
  for (int it = 0; it < max_iter; it++) {
    double ws = 0.0, wv = 0.0;
    for (size_t i = threadIdx.x; i < n; i += kT) {
      const float v = img[box_index(b, i, W, H)];
      const double d = (double)(v - mean);
      const float w = (float)exp(-(d * d) / (2.0 * (double)var));
      ws += (double)w;
      wv += (double)(w * v);
    }
    ws = cta_sum(ws, s);
    wv = cta_sum(wv, s);
    const float prev = mean;
    if (threadIdx.x == 0) smean = (float)(wv / fmax(ws, (double)kEps));
    __syncthreads();
    mean = smean;
    __syncthreads();
    if (!(fabsf(mean - prev) > 1e-5f)) break;
  }
  if (threadIdx.x == 0) out[blockIdx.x] = mean;
}

// Least-trimmed-squares variance of each leaf (QuadTree_.calculateLTSVariance):
// the mean of the h = floor(frac n) smallest squared residuals (v - robust
// mean)^2, over h + eps. The h-th smallest is found by a radix select on the
// float bits (non-negative floats order as unsigned integers), then the sum
// of everything below it plus the ties it takes.
__global__ void __launch_bounds__(kTreeThreads)
    k_tree_lts(const float* __restrict__ img, int W, int H, const TreeBox* __restrict__ boxes,
               const float* __restrict__ means, float frac, float* __restrict__ out) {
  __shared__ double s[kT];
  __shared__ unsigned hist[256];
  __shared__ unsigned sel_prefix, sel_k;
  const TreeBox b = boxes[blockIdx.x];
  const size_t n = (size_t)b.w * b.h * b.d;
  const float m = means[blockIdx.x];
  const int h = (int)floorf(frac * (float)n);
  if (h <= 0) {
    if (threadIdx.x == 0) out[blockIdx.x] = 0.0f;
    return;
  }
  if (threadIdx.x == 0) {
    sel_prefix = 0u;
    sel_k = (unsigned)h;  // rank (1-based) of the value to find
  }
  unsigned mask = 0u;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += kT) hist[i] = 0u;
    __syncthreads();
    const unsigned prefix = sel_prefix;
    for (size_t i = threadIdx.x; i < n; i += kT) {
      const float d = img[box_index(b, i, W, H)] - m;
      const unsigned u = __float_as_uint(d * d);
      if ((u & mask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned k = sel_k, dgt = 0;
      for (; dgt < 255; dgt++) {
        if (hist[dgt] >= k) break;
        k -= hist[dgt];
      }
      sel_prefix = prefix | (dgt << shift);
      sel_k = k;
    }
    mask |= 255u << shift;
    __syncthreads();
  }
  const unsigned tbits = sel_prefix;
  const float t = __uint_as_float(tbits);
  double below = 0.0, cnt = 0.0;
  for (size_t i = threadIdx.x; i < n; i += kT) {
    const float d = img[box_index(b, i, W, H)] - m;
    const float r = d * d;
    if (__float_as_uint(r) < tbits) {
      below += (double)r;
      cnt += 1.0;
    }
  }
  below = cta_sum(below, s);
  cnt = cta_sum(cnt, s);
  if (threadIdx.x == 0) {
    const double sum = below + ((double)h - cnt) * (double)t;
    out[blockIdx.x] = (float)(sum / (double)((float)h + kEps));
  }
}

}  // namespace sred
