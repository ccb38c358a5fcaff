// 3D (volume) block repetition maps: local statistics and one reference
// block against every interior block of a volume, with the host steps of
// java/CLUtils.java:1133-1637 (metric transform, relevance mask,
// normalisation) on the device.
//
// FP32 in the reference kernels' evaluation order (cl/kernelGetLocalStatistics3D.cl,
// cl/kernelGetBlock{Pearson,Ssim,Nrmse,AbsDiffStds}3D.cl); compiled with
// -fmad=false so that no multiply-add is fused. One thread per voxel, threads
// of a warp on consecutive x so that every gather of the block is coalesced;
// the block offsets (and reference voxels) sit in shared memory and the
// Pearson chain re-reads the block through L1 instead of holding it in a
// local array.
#include <float.h>

#include "volume.cuh"

namespace sred {

namespace {

__device__ __forceinline__ bool interior3(int x, int y, int z, const Vol3& v) {
  return x >= v.rw && x < v.W - v.rw && y >= v.rh && y < v.H - v.rh && z >= v.rd && z < v.D - v.rd;
}

// Voxel of this thread for the (32, 4) block and ((W+31)/32, (H+3)/4, D) grid
// (or a grid of fewer slices starting at slice v.z0).
__device__ __forceinline__ bool voxel(const Vol3& v, int* x, int* y, int* z, size_t* p) {
  *x = blockIdx.x * blockDim.x + threadIdx.x;
  *y = blockIdx.y * blockDim.y + threadIdx.y;
  *z = blockIdx.z + v.z0;
  if (*x >= v.W || *y >= v.H) return false;
  *p = ((size_t)*z * v.H + *y) * v.W + *x;
  return true;
}

// Order-preserving key of a float for atomicMin/atomicMax on unsigned ints
// (-0 orders below +0, as Math.min / Math.max do).
__device__ __forceinline__ unsigned f2key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key2f(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

}  // namespace

__global__ void __launch_bounds__(128)
    k_local_stats3d(const float* __restrict__ img, Vol3 v, const int* __restrict__ off, float* __restrict__ means,
                    float* __restrict__ stds) {
  extern __shared__ int s_off[];
  for (int i = threadIdx.y * blockDim.x + threadIdx.x; i < v.k; i += blockDim.x * blockDim.y) s_off[i] = off[i];
  __syncthreads();
  int x, y, z;
  size_t p;
  if (!voxel(v, &x, &y, &z, &p)) return;
  if (!interior3(x, y, z, v)) {
    means[p] = 0.0f;
    stds[p] = 0.0f;
    return;
  }
  const float* c = img + p;
  const int K = v.k;
  float mean = 0.0f;
  for (int i = 0; i < K; i++) mean += c[s_off[i]];
  mean /= (float)K;
  float var = 0.0f;
  for (int i = 0; i < K; i++) {
    const float d = c[s_off[i]] - mean;
    var += d * d;
  }
  means[p] = mean;
  stds[p] = sqrtf(var / (float)(K - 1));
}

template <bool CACHE>
__global__ void __launch_bounds__(128)
    k_block_map3d_t(const float* __restrict__ img, Vol3 v, const int* __restrict__ off,
                    const float* __restrict__ ref, float ref_mean, float ref_std, int metric,
                    const float* __restrict__ means, const float* __restrict__ stds, float* __restrict__ out) {
  extern __shared__ int s_off[];
  float* s_ref = reinterpret_cast<float*>(s_off + v.k);
  float* s_t = s_ref + v.k;  // CACHE: [K][128] normalised block values of the Pearson chain
  for (int i = threadIdx.y * blockDim.x + threadIdx.x; i < v.k; i += blockDim.x * blockDim.y) {
    s_off[i] = off[i];
    s_ref[i] = ref[i];
  }
  __syncthreads();
  int x, y, z;
  size_t p;
  if (!voxel(v, &x, &y, &z, &p)) return;
  if (!interior3(x, y, z, v)) {
    out[p] = 0.0f;
    return;
  }
  const float tstd = stds[p];
  const float* c = img + p;
  const int K = v.k;
  if (metric == kAbsDiff) {  // cl/kernelGetBlockAbsDiffStds3D.cl
    out[p] = fabsf(ref_std - tstd);
    return;
  }
  const float tmean = means[p];
  if (metric == kPearson) {
    // cl/kernelGetBlockPearson3D.cl: min-max of the block, minus its mean,
    // min-max again, then the covariance with the reference. Every division of
    // a pass shares its divisor (div_fixed: correctly rounded, as the
    // kernel's own divisions); with CACHE the first normalisation is kept in
    // shared memory for the last pass instead of being computed again.
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int i = 0; i < K; i++) {
      const float t = c[s_off[i]];
      mn = fminf(mn, t);
      mx = fmaxf(mx, t);
    }
    const float d1 = mx - mn + kEps, y1 = __frcp_rn(d1);
    float mn2 = FLT_MAX, mx2 = -FLT_MAX;
    for (int i = 0; i < K; i++) {
      const float t = div_fixed(c[s_off[i]] - mn, d1, y1) - tmean;
      if (CACHE) s_t[i * 128 + tid] = t;
      mn2 = fminf(mn2, t);
      mx2 = fmaxf(mx2, t);
    }
    const float d2 = mx2 - mn2 + kEps, y2 = __frcp_rn(d2);
    float cov = 0.0f;
    for (int i = 0; i < K; i++) {
      const float t = CACHE ? s_t[i * 128 + tid] : div_fixed(c[s_off[i]] - mn, d1, y1) - tmean;
      cov += s_ref[i] * div_fixed(t - mn2, d2, y2);
    }
    cov /= (float)(K - 1);
    if (ref_std == 0.0f && tstd == 0.0f) out[p] = 1.0f;
    else if (ref_std == 0.0f || tstd == 0.0f) out[p] = 0.0f;
    else out[p] = fmaxf(0.0f, cov / ((ref_std * tstd) + kEps));
    return;
  }
  if (metric == kSsim) {  // cl/kernelGetBlockSsim3D.cl
    float cov = 0.0f;
    for (int i = 0; i < K; i++) cov += s_ref[i] * (c[s_off[i]] - tmean);
    cov /= (float)(K - 1);
    if (ref_std == 0.0f && tstd == 0.0f) {
      out[p] = 1.0f;
    } else if (ref_std == 0.0f || tstd == 0.0f) {
      out[p] = 0.0f;
    } else {
      const float ssim = ((2.0f * ref_mean * tmean + kC1) * (2.0f * cov + kC2)) /
                         (((ref_mean * ref_mean) + (tmean * tmean) + kC1) * ((ref_std * ref_std) + (tstd * tstd) + kC2));
      out[p] = fmaxf(0.0f, ssim);
    }
    return;
  }
  // NRMSE, cl/kernelGetBlockNrmse3D.cl
  float mse = 0.0f;
  for (int i = 0; i < K; i++) {
    const float d = s_ref[i] - (c[s_off[i]] - tmean);
    mse += d * d;
  }
  mse /= (float)K;
  out[p] = sqrtf(mse);
}

cudaError_t launch_block_map3d(const float* img, Vol3 v, const int* off, const float* ref, float ref_mean,
                               float ref_std, int metric, const float* means, const float* stds, float* out,
                               cudaStream_t st, int z1) {
  const dim3 grid((v.W + 31) / 32, (v.H + 3) / 4, (z1 < 0 ? v.D : z1) - v.z0), blk(32, 4);
  // The Pearson chain caches its first normalisation (K x 128 floats) while
  // that fits in 96 KB of shared memory; past it, it recomputes.
  const size_t smem_base = 2 * sizeof(int) * (size_t)v.k;
  const size_t smem_cache = smem_base + sizeof(float) * 128 * (size_t)v.k;
  if (metric == kPearson && smem_cache <= 96 * 1024) {
    if (smem_cache > 48 * 1024) {
      const cudaError_t e =
          cudaFuncSetAttribute(k_block_map3d_t<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cache);
      if (e != cudaSuccess) return e;
    }
    k_block_map3d_t<true><<<grid, blk, smem_cache, st>>>(img, v, off, ref, ref_mean, ref_std, metric, means, stds,
                                                         out);
  } else {
    k_block_map3d_t<false><<<grid, blk, smem_base, st>>>(img, v, off, ref, ref_mean, ref_std, metric, means, stds,
                                                          out);
  }
  return cudaGetLastError();
}

// Elementwise a[i] / b by div_fixed (diagnostics: checked against IEEE division).
__global__ void k_divide_fixed(const float* __restrict__ a, size_t n, float b, float* __restrict__ out) {
  const float y = __frcp_rn(b);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = div_fixed(a[i], b, y);
}

// Elementwise a[i] / b by the FP64 div_fixed (diagnostics: checked against IEEE division).
__global__ void k_divide_fixed64(const double* __restrict__ a, size_t n, double b, double* __restrict__ out) {
  const double y = __drcp_rn(b);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = div_fixed(a[i], b, y);
}

// Host steps on the interior (java/CLUtils.java:1459-1471, 1590-1600): NRMSE
// inverted (0 -> 1), Abs-diff turned into 1 - x.
__global__ void k_block3d_post(float* __restrict__ a, Vol3 v, int metric) {
  int x, y, z;
  size_t p;
  if (!voxel(v, &x, &y, &z, &p) || !interior3(x, y, z, v)) return;
  if (metric == kNrmse) a[p] = a[p] == 0.0f ? 1.0f : 1.0f / a[p];
  else if (metric == kAbsDiff) a[p] = 1.0f - a[p];
}

// java/Utils.java:1501-1525 (getRelevanceMask3D) for the threshold
// noise_var * c; map (if not null) is multiplied by the mask (applyMask3D).
__global__ void k_mask3d(const float* __restrict__ stds, Vol3 v, float thr, float* __restrict__ mask,
                         float* __restrict__ map) {
  int x, y, z;
  size_t p;
  if (!voxel(v, &x, &y, &z, &p)) return;
  float m = 0.0f;
  if (interior3(x, y, z, v)) m = (stds[p] * stds[p]) <= thr ? 0.0f : 1.0f;
  mask[p] = m;
  if (map) map[p] *= m;
}

// java/Utils.java:1572-1630 (normalizeImage3D): min and max over the interior
// (where mask > 0 when a mask is given); mm = {min key, max key}. Grid-stride
// over the volume (a grid of a few CTAs per SM) so that each warp issues one
// pair of atomics for many voxels.
__global__ void k_minmax3d(const float* __restrict__ a, const float* __restrict__ mask, Vol3 v,
                           unsigned* __restrict__ mm) {
  const size_t n = (size_t)v.W * v.H * v.D, plane = (size_t)v.W * v.H;
  unsigned lo = 0xffffffffu, hi = 0u;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(p / plane), y = (int)((p % plane) / v.W), x = (int)(p % v.W);
    if (interior3(x, y, z, v) && (!mask || mask[p] > 0.0f)) {
      const unsigned k = f2key(a[p]);
      lo = min(lo, k);
      hi = max(hi, k);
    }
  }
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0 && lo != 0xffffffffu) {
    atomicMin(mm, lo);
    atomicMax(mm + 1, hi);
  }
}

__global__ void k_remap3d(float* __restrict__ a, const float* __restrict__ mask, Vol3 v,
                          const unsigned* __restrict__ mm) {
  if (mm[0] == 0xffffffffu) return;  // no voxel selected: the reference changes nothing
  int x, y, z;
  size_t p;
  if (!voxel(v, &x, &y, &z, &p) || !interior3(x, y, z, v) || (mask && !(mask[p] > 0.0f))) return;
  const float mn = key2f(mm[0]), mx = key2f(mm[1]);
  a[p] = (a[p] - mn) / (mx - mn + kEps);
}

// ---------------------------------------------------------------------------
// 3D global repetition map: flags, operand packing and finalisation around
// the 2D pair engines (cl/kernelGetGlobal*3D.cl, java/CLUtils.java:2225-2790).
// ---------------------------------------------------------------------------

// mask: sigma^2 > threshold on the interior (getRelevanceMask3D).
// flags: 1 = reference and test block (interior, !(sigma^2 < threshold),
// sigma^2 != 0: the 3D kernels skip a reference voxel of zero variance);
// 2 = test block only, sigma == 0 (a flat block still counts as a test block
// of Pearson, SSIM and NRMSE; flat_columns = 0 drops it, as Abs-diff does).
// A voxel with sigma != 0 but sigma^2 == 0 (sigma below 1.1e-23) is neither;
// the reference would still use it as a test block.
// n_mask counts mask > 0 (the command's nPixels).
__global__ void k_flags3d(const float* __restrict__ stds, Vol3 v, float thr, int flat_columns,
                          float* __restrict__ mask, uint8_t* __restrict__ flags,
                          unsigned long long* __restrict__ n_mask) {
  const size_t n = (size_t)v.W * v.H * v.D, plane = (size_t)v.W * v.H;
  unsigned c = 0;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    const int z = (int)(p / plane), y = (int)((p % plane) / v.W), x = (int)(p % v.W);
    const bool in = interior3(x, y, z, v);
    const float s = stds[p];
    const float s2 = s * s;
    const float m = (in && !(s2 <= thr)) ? 1.0f : 0.0f;
    mask[p] = m;
    uint8_t f = 0;
    if (in && !(s2 < thr)) {
      if (s2 != 0.0f) f = 1;
      else if (s == 0.0f && flat_columns) f = 2;
    }
    flags[p] = f;
    c += m > 0.0f ? 1u : 0u;
  }
  const unsigned wc = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && wc) atomicAdd(n_mask, (unsigned long long)wc);
}

// One warp per listed block: FP64 moments of its ellipsoid vector, the unit
// vector (x - mu) / |x - mu| as FP32 (mode 0, row pitch kp) or as the two- /
// three-level split BF16 operands (mode 1 / 2, store_split, row pitch kq),
// and the epilogue parameters; the same quantities as the 2D packing, over
// linear offsets.
__global__ void k_pack3d(const float* __restrict__ img, Vol3 v, const int* __restrict__ off,
                         const int* __restrict__ gram_pix, int n, float wscale, int mode, float* __restrict__ U,
                         int kp, __nv_bfloat16* __restrict__ A, __nv_bfloat16* __restrict__ B, int kq,
                         BlockParams* __restrict__ params, float* __restrict__ tile_rmax) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int K = v.k;
  for (int j = gw; j < n; j += nw) {
    const float* c = img + (size_t)gram_pix[j];
    double s = 0.0;
    for (int i = lane; i < K; i += 32) s += (double)c[off[i]];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double mu = s / K;
    double var = 0.0;
    for (int i = lane; i < K; i += 32) {
      const double d = (double)c[off[i]] - mu;
      var += d * d;
    }
    for (int o = 16; o; o >>= 1) var += __shfl_xor_sync(0xffffffffu, var, o);
    const double nrm = sqrt(var);
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    const double sigma = sqrt(var / (K - 1));
    for (int i = lane; i < K; i += 32) {
      const double u = ((double)c[off[i]] - mu) * inv;
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
    if (lane == 0) {
      BlockParams bp;
      bp.a = (float)(sigma * (double)wscale);
      bp.e = sigma > 0.0 ? (float)((double)kEps / sigma) : 0.0f;
      bp.r = sigma > 0.0 ? (float)(1.0 / sigma) : 0.0f;
      bp.sigma = (float)sigma;
      bp.mu = (float)mu;
      bp.pad0 = bp.pad1 = bp.pad2 = 0.0f;
      params[j] = bp;
      atomicMax(reinterpret_cast<int*>(tile_rmax) + (j >> 7), __float_as_int(bp.r));
    }
  }
}

// num / (den nPixels + eps) in FP64 over the interior, with the flat test
// blocks' closed-form share: n_flat pairs of weight 2^-(a_p^2) each, and for
// NRMSE a term sqrt((K-1)/K) sigma_p per pair times that weight (the flat
// block's centred vector is zero). NRMSE and Abs-diff are then inverted where
// mask > 0 (the FP32 value; 0 -> 1), and the mask applied when apply_mask.
__global__ void k_finalize3d(const int* __restrict__ slot, Vol3 v, const double* __restrict__ num,
                             const double* __restrict__ den, const BlockParams* __restrict__ params, int n_flat,
                             int metric, double sk, double n_pixels, const float* __restrict__ mask, int apply_mask,
                             float* __restrict__ out) {
  int x, y, z;
  size_t p;
  if (!voxel(v, &x, &y, &z, &p)) return;
  float o = 0.0f;
  if (interior3(x, y, z, v)) {
    const int s = slot[p];
    double nu = 0.0, de = 0.0;
    if (s >= 0) {
      const BlockParams bp = params[s];
      const double a = (double)bp.a;
      const double w0 = exp2(-(a * a));
      nu = num[s];
      de = den[s] + (double)n_flat * w0;
      if (metric == kNrmse) nu += (double)n_flat * sk * (double)bp.sigma * w0;
    }
    o = (float)(nu / (de * n_pixels + (double)kEps));
    if ((metric == kNrmse || metric == kAbsDiff) && mask[p] > 0.0f) o = (o == 0.0f) ? 1.0f : 1.0f / o;
    if (apply_mask) o *= mask[p];
  }
  out[p] = o;
}

int build_ellipsoid(int bw, int bh, int bd, int W, int H, int* off) {
  const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
  int k = 0;
  for (int z = -rd; z <= rd; z++)
    for (int y = -rh; y <= rh; y++)
      for (int x = -rw; x <= rw; x++) {
        const float fx = (float)x, fy = (float)y, fz = (float)z;
        if (((fx * fx) / (float)(rw * rw)) + ((fy * fy) / (float)(rh * rh)) + ((fz * fz) / (float)(rd * rd)) <=
            1.0f) {
          if (off && k < kMaxK3) off[k] = z * W * H + y * W + x;
          k++;
        }
      }
  return k;
}

}  // namespace sred
