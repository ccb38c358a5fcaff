// Redundancy classification (java/ClassifyRedundancy_.java): k-means++ with
// Lloyd iterations over the interior values of a map, the algorithm of the
// reference's clusterer (commons-math3 3.6.1 KMeansPlusPlusClusterer, maximum
// 1000 iterations, Euclidean distance, an empty cluster refilled from the
// cluster of largest distance variance).
//
// The per-point work runs here; the few per-iteration decisions (sampling the
// next centre, new centres from the block sums) run on the host. Every sum is
// taken in one fixed order, so a run is deterministic: block b covers points
// [b * kKmSpan, (b + 1) * kKmSpan); thread t adds points b * kKmSpan + j *
// kKmThreads + t for j = 0..kKmPer-1 in turn; the 256 thread values are then
// added pairwise (t += t + 128, t += t + 64, ..., t += t + 1).
#include "cluster.cuh"

namespace sred {

namespace {

// Fixed-order block sum of one double per thread into out (thread 0 writes).
__device__ __forceinline__ void block_sum_fixed(double v, double* s, double* out) {
  s[threadIdx.x] = v;
  __syncthreads();
  for (int stride = kKmThreads / 2; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) s[threadIdx.x] += s[threadIdx.x + stride];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
  __syncthreads();
}

}  // namespace

// Interior values of the map as double, raster order.
__global__ void k_km_gather(const float* __restrict__ map, int W, int H, int border, double* __restrict__ x) {
  const int iw = W - 2 * border;
  const size_t n = (size_t)iw * (H - 2 * border);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t y = i / iw + border, xx = i % iw + border;
    x[i] = (double)map[y * W + xx];
  }
}

// k-means++ seeding step: d2[i] = (x_i - c)^2 (first) or min(d2[i], (x_i - c)^2),
// and the fixed-order block sums of d2.
__global__ void __launch_bounds__(kKmThreads)
    k_km_d2(const double* __restrict__ x, size_t n, double c, int first, double* __restrict__ d2,
            double* __restrict__ partial) {
  __shared__ double s[kKmThreads];
  const size_t base = (size_t)blockIdx.x * kKmSpan;
  double v = 0.0;
  for (int j = 0; j < kKmPer; j++) {
    const size_t i = base + (size_t)j * kKmThreads + threadIdx.x;
    if (i < n) {
      const double d = x[i] - c;
      const double e = d * d;
      const double m = first ? e : fmin(d2[i], e);
      d2[i] = m;
      v += m;
    }
  }
  block_sum_fixed(v, s, partial + blockIdx.x);
}

// Lloyd assignment: nearest centre (first of equals), the number of points
// whose cluster changed, and the fixed-order block sums per cluster of the
// values, the counts and the squared distances to the assigned centre.
// bsum/bcnt: [blocks][k]; bwcss: [blocks].
__global__ void __launch_bounds__(kKmThreads)
    k_km_assign(const double* __restrict__ x, size_t n, const double* __restrict__ centers, int k,
                int* __restrict__ labels, unsigned long long* __restrict__ changed, double* __restrict__ bsum,
                double* __restrict__ bcnt, double* __restrict__ bwcss) {
  __shared__ double s[kKmThreads];
  __shared__ double cs[kKmMaxK];
  if (threadIdx.x < k) cs[threadIdx.x] = centers[threadIdx.x];
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kKmSpan;
  double xv[kKmPer];
  int lab[kKmPer];
  double w = 0.0;
  unsigned ch = 0;
  for (int j = 0; j < kKmPer; j++) {
    const size_t i = base + (size_t)j * kKmThreads + threadIdx.x;
    lab[j] = -1;
    xv[j] = 0.0;
    if (i < n) {
      const double v = x[i];
      int best = 0;
      double bd = (v - cs[0]) * (v - cs[0]);
      for (int c = 1; c < k; c++) {
        const double d = (v - cs[c]) * (v - cs[c]);
        if (d < bd) {
          bd = d;
          best = c;
        }
      }
      if (labels[i] != best) ch++;
      labels[i] = best;
      lab[j] = best;
      xv[j] = v;
      w += bd;
    }
  }
  const unsigned wc = __reduce_add_sync(0xffffffffu, ch);
  if ((threadIdx.x & 31) == 0 && wc) atomicAdd(changed, (unsigned long long)wc);
  block_sum_fixed(w, s, bwcss + blockIdx.x);
  for (int c = 0; c < k; c++) {
    double sv = 0.0, sc = 0.0;
    for (int j = 0; j < kKmPer; j++)
      if (lab[j] == c) {
        sv += xv[j];
        sc += 1.0;
      }
    block_sum_fixed(sv, s, bsum + (size_t)blockIdx.x * k + c);
    block_sum_fixed(sc, s, bcnt + (size_t)blockIdx.x * k + c);
  }
}

// For the empty-cluster rule: fixed-order block sums per cluster of the
// distances |x - c_label| and of their squares (the variance follows on the
// host).
__global__ void __launch_bounds__(kKmThreads)
    k_km_distvar(const double* __restrict__ x, size_t n, const double* __restrict__ centers, int k,
                 const int* __restrict__ labels, double* __restrict__ bd1, double* __restrict__ bd2) {
  __shared__ double s[kKmThreads];
  __shared__ double cs[kKmMaxK];
  if (threadIdx.x < k) cs[threadIdx.x] = centers[threadIdx.x];
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kKmSpan;
  for (int c = 0; c < k; c++) {
    double a = 0.0, b = 0.0;
    for (int j = 0; j < kKmPer; j++) {
      const size_t i = base + (size_t)j * kKmThreads + threadIdx.x;
      if (i < n && labels[i] == c) {
        const double d = fabs(x[i] - cs[c]);
        a += d;
        b += d * d;
      }
    }
    block_sum_fixed(a, s, bd1 + (size_t)blockIdx.x * k + c);
    block_sum_fixed(b, s, bd2 + (size_t)blockIdx.x * k + c);
  }
}

// Output map: the cluster rank of each interior point (0 = the largest
// cluster); the border stays 0, as the reference's int[] starts.
__global__ void k_km_scatter(const int* __restrict__ labels, const int* __restrict__ rank, int W, int H, int border,
                             float* __restrict__ out) {
  const size_t total = (size_t)W * H;
  const int iw = W - 2 * border;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(p / W), x = (int)(p % W);
    float v = 0.0f;
    if (x >= border && x < W - border && y >= border && y < H - border)
      v = (float)rank[labels[(size_t)(y - border) * iw + (x - border)]];
    out[p] = v;
  }
}

}  // namespace sred
