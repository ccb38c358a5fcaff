// Relevance-mask tools: the relevance mask of one filter constant
// (java/RelevanceMask2D_.java), a stack of masks over a range of constants
// (java/RelevanceMaskStack2D_.java) and the range of constants between an
// all-relevant and an all-irrelevant mask (java/OptimiseRelevanceMask_.java).
//
// All three compare a per-pixel block statistic s, squared, against a
// threshold: s is the local standard deviation (cl/kernelGetLocalMeans.cl) in
// the first tool and the local variance (cl/kernelGetRelevanceMask2D.cl,
// stored in a buffer the Java code calls localStds and squares) in the other
// two. FP32 in the kernels' order; compiled with -fmad=false.
#include "common.cuh"
#include "relevance.cuh"

namespace sred {

// cl/kernelGetRelevanceMask2D.cl (take_sqrt = 0) and cl/kernelGetLocalMeans.cl
// (take_sqrt = 1): the ellipse block's mean (sequential sum / K) and the
// (K-1) variance, or its square root; border pixels 0.
__global__ void k_local_var2d(const float* __restrict__ img, int W, int H, Ellipse e, int take_sqrt,
                              float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= W) return;
  const size_t p = (size_t)y * W + x;
  if (x < e.rw || x >= W - e.rw || y < e.rh || y >= H - e.rh) {
    out[p] = 0.0f;
    return;
  }
  float mean = 0.0f;
  for (int i = 0; i < e.k; i++) mean += img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])];
  mean /= (float)e.k;
  float var = 0.0f;
  for (int i = 0; i < e.k; i++) {
    const float d = img[(size_t)(y + e.dy[i]) * W + (x + e.dx[i])] - mean;
    var += d * d;
  }
  var /= (float)(e.k - 1);
  out[p] = take_sqrt ? sqrtf(var) : var;
}

// Noise tiles with FP64 sums (the getMeanAndVarBlock of
// java/RelevanceMask2D_.java): mean and sum of squares in double over the
// float pixels (each square a float product), var = sq / n - mean^2 in
// double, stored as float.
__global__ void k_noise_tiles64(const float* __restrict__ img, int W, int t, int nbx, int nb,
                                float* __restrict__ vars) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int bx = i % nbx, by = i / nbx;
  double mean = 0.0, sq = 0.0;
  for (int y = by * t; y < (by + 1) * t; y++)
    for (int x = bx * t; x < (bx + 1) * t; x++) {
      const float v = img[(size_t)y * W + x];
      mean += (double)v;
      sq += (double)(v * v);
    }
  const int n = t * t;
  mean = mean / n;
  vars[i] = (float)(sq / n - mean * mean);
}

// Masks of n thresholds (one per blockIdx.y): 1 where the interior pixel's
// s^2 is neither below the threshold nor 0, else 0.
__global__ void k_sweep_masks(const float* __restrict__ stat, int W, int H, int rw, int rh,
                              const float* __restrict__ thr, float* __restrict__ masks) {
  const size_t n = (size_t)W * H;
  const float t = thr[blockIdx.y];
  float* m = masks + n * blockIdx.y;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    float v = 0.0f;
    if (!(x < rw || x >= W - rw || y < rh || y >= H - rh)) {
      const float s2 = stat[p] * stat[p];
      v = (s2 < t || s2 == 0.0f) ? 0.0f : 1.0f;
    }
    m[p] = v;
  }
}

// Smallest and largest s^2 over the interior, as the bit patterns of the
// non-negative floats (which order like unsigned integers); mm = {min, max}.
__global__ void k_stat_sq_minmax(const float* __restrict__ stat, int W, int H, int rw, int rh,
                                 unsigned* __restrict__ mm) {
  const size_t n = (size_t)W * H;
  unsigned lo = 0xffffffffu, hi = 0u;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    if (x < rw || x >= W - rw || y < rh || y >= H - rh) continue;
    const unsigned b = __float_as_uint(stat[p] * stat[p]);
    lo = min(lo, b);
    hi = max(hi, b);
  }
  lo = __reduce_min_sync(0xffffffffu, lo);
  hi = __reduce_max_sync(0xffffffffu, hi);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}

}  // namespace sred
