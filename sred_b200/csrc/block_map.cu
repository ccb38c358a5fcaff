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

constexpr int kTileX = 32, kTileY = 16, kThreadsY = 8;  // each thread: rows y and y + 8 of the tile

// The metric of one pixel from its block sums (reference order, explicitly
// rounded), and its local std.
__device__ __forceinline__ float block_metric_value(int metric, int K, float mean, float v, float acc, float rr,
                                                    float xx, float ref_mean, float ref_std, float* sd_out) {
  const float sd = __fsqrt_rn(__fdiv_rn(v, (float)(K - 1)));
  *sd_out = sd;
  if (metric == kAbsDiff) return fabsf(__fsub_rn(ref_std, sd));
  if (metric == kNrmse) return __fsqrt_rn(__fdiv_rn(acc, (float)K));
  if (metric == kCosine) return __fdiv_rn(acc, __fadd_rn(__fmul_rn(__fsqrt_rn(rr), __fsqrt_rn(xx)), kEps));
  const float cov = __fdiv_rn(acc, (float)(K - 1));
  if (ref_std == 0.0f && sd == 0.0f) return 1.0f;
  if (ref_std == 0.0f || sd == 0.0f) return 0.0f;
  if (metric == kPearson) return fmaxf(0.0f, __fdiv_rn(cov, __fadd_rn(__fmul_rn(ref_std, sd), kEps)));
  // SSIM, textbook sum form (cl/kernelGetBlockSsim2D.cl:79)
  const float a = __fadd_rn(__fmul_rn(__fmul_rn(2.0f, ref_mean), mean), kC1);
  const float b = __fadd_rn(__fmul_rn(2.0f, cov), kC2);
  const float cc = __fadd_rn(__fadd_rn(__fmul_rn(ref_mean, ref_mean), __fmul_rn(mean, mean)), kC1);
  const float dd = __fadd_rn(__fadd_rn(__fmul_rn(ref_std, ref_std), __fmul_rn(sd, sd)), kC2);
  return fmaxf(0.0f, __fdiv_rn(__fmul_rn(a, b), __fmul_rn(cc, dd)));
}

__global__ void __launch_bounds__(kTileX* kThreadsY)
    k_block_map(const float* __restrict__ img_all, int W, int H, int frames, Ellipse e, RefBlock rb,
                int metric, float* __restrict__ out_all, float* __restrict__ stds_out) {
  // shared: the image tile (kTileY + 2rh) x (kTileX + 2rw), then the ellipse
  // as linear tile offsets (K ints) and the reference block (K floats). Each
  // thread evaluates two pixels, rows y and y + 8, so every broadcast load of
  // an offset or a reference value serves both; each pixel keeps the
  // reference's sequential order.
  extern __shared__ float tile[];
  const int f = blockIdx.z;
  const float* img = img_all + (size_t)f * W * H;
  float* out = out_all + (size_t)f * W * H;
  const int tw = kTileX + 2 * e.rw, th = kTileY + 2 * e.rh;
  int* s_off = reinterpret_cast<int*>(tile + tw * th);
  float* s_ref = reinterpret_cast<float*>(s_off + e.k);
  const int x0 = blockIdx.x * kTileX - e.rw, y0 = blockIdx.y * kTileY - e.rh;
  const int tid = threadIdx.y * kTileX + threadIdx.x;
  for (int i = tid; i < tw * th; i += kTileX * kThreadsY) {
    const int ty = i / tw, tx = i - ty * tw;
    const int gx = x0 + tx, gy = y0 + ty;
    tile[i] = (gx >= 0 && gx < W && gy >= 0 && gy < H) ? img[(size_t)gy * W + gx] : 0.0f;
  }
  for (int i = tid; i < e.k; i += kTileX * kThreadsY) {
    s_off[i] = e.dy[i] * tw + e.dx[i];
    s_ref[i] = rb.px[i];
  }
  __syncthreads();
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int ya = blockIdx.y * kTileY + threadIdx.y, yb = ya + kThreadsY;
  if (x >= W || ya >= H) return;
  const bool has_b = yb < H;
  const bool in_x = x >= e.rw && x < W - e.rw;
  const bool in_a = in_x && ya >= e.rh && ya < H - e.rh;
  const bool in_b = has_b && in_x && yb >= e.rh && yb < H - e.rh;
  const size_t pa = (size_t)ya * W + x, pb = (size_t)yb * W + x;
  if (!in_a && !in_b) {
    out[pa] = 0.0f;
    if (stds_out) stds_out[(size_t)f * W * H + pa] = 0.0f;
    if (has_b) {
      out[pb] = 0.0f;
      if (stds_out) stds_out[(size_t)f * W * H + pb] = 0.0f;
    }
    return;
  }
  // (a pixel outside the interior is evaluated on the zero-padded tile and
  // discarded)
  const float* ca = tile + (threadIdx.y + e.rh) * tw + (threadIdx.x + e.rw);
  const float* cb = ca + kThreadsY * tw;
  const int K = e.k;
  float sa = 0.0f, sb = 0.0f;
  for (int i = 0; i < K; i++) {
    const int o = s_off[i];
    sa = __fadd_rn(sa, ca[o]);
    sb = __fadd_rn(sb, cb[o]);
  }
  const float ma = __fdiv_rn(sa, (float)K), mb = __fdiv_rn(sb, (float)K);
  float va = 0.0f, aa = 0.0f, ra = 0.0f, xa = 0.0f;
  float vb = 0.0f, ab = 0.0f, rb2 = 0.0f, xb = 0.0f;
  for (int i = 0; i < K; i++) {
    const int o = s_off[i];
    const float ref = s_ref[i];
    const float pxa = ca[o], pxb = cb[o];
    const float da = __fsub_rn(pxa, ma), db = __fsub_rn(pxb, mb);
    va = __fadd_rn(va, __fmul_rn(da, da));
    vb = __fadd_rn(vb, __fmul_rn(db, db));
    if (metric == kNrmse) {
      const float ta = __fsub_rn(ref, da), tb = __fsub_rn(ref, db);
      aa = __fadd_rn(aa, __fmul_rn(ta, ta));
      ab = __fadd_rn(ab, __fmul_rn(tb, tb));
    } else if (metric == kCosine) {
      aa = __fadd_rn(aa, __fmul_rn(ref, pxa));
      ab = __fadd_rn(ab, __fmul_rn(ref, pxb));
      ra = __fadd_rn(ra, __fmul_rn(ref, ref));
      rb2 = __fadd_rn(rb2, __fmul_rn(ref, ref));
      xa = __fadd_rn(xa, __fmul_rn(pxa, pxa));
      xb = __fadd_rn(xb, __fmul_rn(pxb, pxb));
    } else {
      aa = __fadd_rn(aa, __fmul_rn(ref, da));
      ab = __fadd_rn(ab, __fmul_rn(ref, db));
    }
  }
  float sd;
  const float r_a = block_metric_value(metric, K, ma, va, aa, ra, xa, rb.mean, rb.std, &sd);
  out[pa] = in_a ? r_a : 0.0f;
  if (stds_out) stds_out[(size_t)f * W * H + pa] = in_a ? sd : 0.0f;
  if (has_b) {
    const float r_b = block_metric_value(metric, K, mb, vb, ab, rb2, xb, rb.mean, rb.std, &sd);
    out[pb] = in_b ? r_b : 0.0f;
    if (stds_out) stds_out[(size_t)f * W * H + pb] = in_b ? sd : 0.0f;
  }
}

size_t block_map_smem(const Ellipse& e) {
  return sizeof(float) * (size_t)(kTileX + 2 * e.rw) * (kTileY + 2 * e.rh) + (sizeof(int) + sizeof(float)) * (size_t)e.k;
}

void block_map_launch_shape(int w, int h, int frames, dim3* grid, dim3* block) {
  *grid = dim3((w + kTileX - 1) / kTileX, (h + kTileY - 1) / kTileY, frames);
  *block = dim3(kTileX, kThreadsY);
}

__global__ void k_init_minmax(unsigned* mm, int planes) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < planes; i += gridDim.x * blockDim.x) {
    mm[2 * i] = 0xffffffffu;
    mm[2 * i + 1] = 0u;
  }
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
