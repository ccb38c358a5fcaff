// Block ("local") repetition map: one reference block against every interior
// block of an image (or of each frame of a stack).
//
// One streaming pass per pixel fuses the block moments with the metric: the
// kernel reads only the image and writes only the map (plus, optionally, the
// local stds the relevance mask needs). The moments and the metric follow the
// reference kernels' FP32 evaluation order with explicitly rounded operations,
// so the raw map equals the reference's (cl/kernelGetBlock{Pearson,Ssim,
// Nrmse,AbsDiffStds}2D.cl, with cl/kernelGetLocalStatistics2D.cl for the
// moments) bit for bit. The image tile and its halo are staged in shared
// memory so every pixel is read from HBM once.
#include "common.cuh"
#include "kernels.cuh"

namespace sred {

constexpr int kTileX = 32, kTileY = 8;

__global__ void __launch_bounds__(kTileX* kTileY)
    k_block_map(const float* __restrict__ img_all, int W, int H, int frames, Ellipse e, RefBlock rb,
                int metric, float* __restrict__ out_all, float* __restrict__ stds_out) {
  // shared: the image tile (kTileY + 2rh) x (kTileX + 2rw), then the ellipse
  // as linear tile offsets (K ints) and the reference block (K floats), so
  // each element of a pass costs two broadcast shared loads
  extern __shared__ float tile[];
  const int f = blockIdx.z;
  const float* img = img_all + (size_t)f * W * H;
  float* out = out_all + (size_t)f * W * H;
  const int tw = kTileX + 2 * e.rw, th = kTileY + 2 * e.rh;
  int* s_off = reinterpret_cast<int*>(tile + tw * th);
  float* s_ref = reinterpret_cast<float*>(s_off + e.k);
  const int x0 = blockIdx.x * kTileX - e.rw, y0 = blockIdx.y * kTileY - e.rh;
  for (int i = threadIdx.y * kTileX + threadIdx.x; i < tw * th; i += kTileX * kTileY) {
    const int ty = i / tw, tx = i - ty * tw;
    const int gx = x0 + tx, gy = y0 + ty;
    tile[i] = (gx >= 0 && gx < W && gy >= 0 && gy < H) ? img[(size_t)gy * W + gx] : 0.0f;
  }
  for (int i = threadIdx.y * kTileX + threadIdx.x; i < e.k; i += kTileX * kTileY) {
    s_off[i] = e.dy[i] * tw + e.dx[i];
    s_ref[i] = rb.px[i];
  }
  __syncthreads();
  const int x = blockIdx.x * kTileX + threadIdx.x, y = blockIdx.y * kTileY + threadIdx.y;
  if (x >= W || y >= H) return;
  const size_t p = (size_t)y * W + x;
  if (x < e.rw || x >= W - e.rw || y < e.rh || y >= H - e.rh) {
    out[p] = 0.0f;
    if (stds_out) stds_out[(size_t)f * W * H + p] = 0.0f;
    return;
  }
  const float* c = tile + (threadIdx.y + e.rh) * tw + (threadIdx.x + e.rw);
  const int K = e.k;
  float s = 0.0f;
  for (int i = 0; i < K; i++) s = __fadd_rn(s, c[s_off[i]]);
  const float mean = __fdiv_rn(s, (float)K);
  float v = 0.0f, acc = 0.0f, rr = 0.0f, xx = 0.0f;
  for (int i = 0; i < K; i++) {
    const float px = c[s_off[i]];
    const float d = __fsub_rn(px, mean);
    v = __fadd_rn(v, __fmul_rn(d, d));
    const float ref = s_ref[i];
    if (metric == kNrmse) {
      const float t = __fsub_rn(ref, d);
      acc = __fadd_rn(acc, __fmul_rn(t, t));
    } else if (metric == kCosine) {
      acc = __fadd_rn(acc, __fmul_rn(ref, px));
      rr = __fadd_rn(rr, __fmul_rn(ref, ref));
      xx = __fadd_rn(xx, __fmul_rn(px, px));
    } else {
      acc = __fadd_rn(acc, __fmul_rn(ref, d));
    }
  }
  const float sd = __fsqrt_rn(__fdiv_rn(v, (float)(K - 1)));
  if (stds_out) stds_out[(size_t)f * W * H + p] = sd;
  float r;
  if (metric == kAbsDiff) {
    r = fabsf(__fsub_rn(rb.std, sd));
  } else if (metric == kNrmse) {
    r = __fsqrt_rn(__fdiv_rn(acc, (float)K));
  } else if (metric == kCosine) {
    r = __fdiv_rn(acc, __fadd_rn(__fmul_rn(__fsqrt_rn(rr), __fsqrt_rn(xx)), kEps));
  } else {
    const float cov = __fdiv_rn(acc, (float)(K - 1));
    if (rb.std == 0.0f && sd == 0.0f) {
      r = 1.0f;
    } else if (rb.std == 0.0f || sd == 0.0f) {
      r = 0.0f;
    } else if (metric == kPearson) {
      r = fmaxf(0.0f, __fdiv_rn(cov, __fadd_rn(__fmul_rn(rb.std, sd), kEps)));
    } else {  // SSIM, textbook sum form (cl/kernelGetBlockSsim2D.cl:79)
      const float a = __fadd_rn(__fmul_rn(__fmul_rn(2.0f, rb.mean), mean), kC1);
      const float b = __fadd_rn(__fmul_rn(2.0f, cov), kC2);
      const float cc = __fadd_rn(__fadd_rn(__fmul_rn(rb.mean, rb.mean), __fmul_rn(mean, mean)), kC1);
      const float dd = __fadd_rn(__fadd_rn(__fmul_rn(rb.std, rb.std), __fmul_rn(sd, sd)), kC2);
      r = fmaxf(0.0f, __fdiv_rn(__fmul_rn(a, b), __fmul_rn(cc, dd)));
    }
  }
  out[p] = r;
}

__device__ __forceinline__ float ord_to_float(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Abs-diff post-processing, java/CLUtils.java:936-960: min-max over the
// interior with the maximum starting at Float.MIN_VALUE, then 1 - x.
__global__ void k_block_absdiff_post(float* __restrict__ a_all, int W, int H, int rw, int rh, size_t plane,
                                     const unsigned* __restrict__ mm_all) {
  float* a = a_all + plane * blockIdx.y;
  const unsigned* mm = mm_all + 2 * blockIdx.y;
  const float mn = ord_to_float(mm[0]);
  const float mx = fmaxf(ord_to_float(mm[1]), 1.4e-45f);
  const float d = __fadd_rn(__fsub_rn(mx, mn), kEps);
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < (size_t)W * H;
       p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    if (x < rw || x >= W - rw || y < rh || y >= H - rh) continue;
    a[p] = __fsub_rn(1.0f, __fdiv_rn(__fsub_rn(a[p], mn), d));
  }
}

// NRMSE with relevance constant 0: the interior is the mask (java/CLUtils.java:788-797).
__global__ void k_interior_mask(float* __restrict__ mask_all, int W, int H, int rw, int rh, size_t plane) {
  float* mask = mask_all + plane * blockIdx.y;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < (size_t)W * H;
       p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    mask[p] = (x < rw || x >= W - rw || y < rh || y >= H - rh) ? 0.0f : 1.0f;
  }
}

__global__ void k_apply_mask(float* __restrict__ a, const float* __restrict__ mask, size_t n) {
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
    a[p] = __fmul_rn(a[p], mask[p]);
}

// NRMSE inversion on mask > 0, java/CLUtils.java:809-821.
__global__ void k_invert_masked(float* __restrict__ a_all, const float* __restrict__ mask_all, int W, int H,
                                int rw, int rh, size_t plane) {
  float* a = a_all + plane * blockIdx.y;
  const float* mask = mask_all + plane * blockIdx.y;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < (size_t)W * H;
       p += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(p % W), y = (int)(p / W);
    if (x < rw || x >= W - rw || y < rh || y >= H - rh) continue;
    if (mask[p] > 0.0f) a[p] = (a[p] == 0.0f) ? 1.0f : __fdiv_rn(1.0f, a[p]);
  }
}

}  // namespace sred
