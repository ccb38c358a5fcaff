// Shape metrics: Hu moments and phase correlation (kernels and host helpers).
//
// This file is compiled with -fmad=false: the Hu kernels restate the
// reference's FP32/FP64 evaluation order statement for statement, and a fused
// multiply-add would round differently.
#include <float.h>

#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "shape.cuh"

namespace sred {

// ---------------------------------------------------------------------------
// Hu patch map: kernelGetPatchHu2D.cl:18-267 (FP64), one thread per pixel.
// stds_out (optional): the pixel's FP32 local standard deviation, which the
// relevance mask of the block-map form needs.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_patch_hu(const float* __restrict__ img_all, int W, int H, Ellipse e, int patch_size, double ref_hu1,
               float* __restrict__ out_all, float* __restrict__ stds_out) {
  const size_t plane = (size_t)W * H;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= plane) return;
  const size_t off = (size_t)blockIdx.y * plane;
  const float* img = img_all + off;
  float* out = out_all + off;
  const int x = (int)(idx % W), y = (int)(idx / W), rw = e.rw, rh = e.rh;
  if (x < rw || x >= W - rw || y < rh || y >= H - rh) {
    out[idx] = 0.0f;
    if (stds_out) stds_out[off + idx] = 0.0f;
    return;
  }
  if (stds_out) {
    float m, sd;
    block_stats_f32(img + idx, W, e, &m, &sd);
    stds_out[off + idx] = sd;
  }
  // :129-140: the gather's ellipse test divides integers, which keeps every
  // position of the square except its four corners; the sum is divided by
  // patch_size all the same.
  // (i / rw and j / rh are 0 inside and +-1 on the square's edges, so the
  // test fails exactly where both are +-1; tested that way, in the same order)
  double mean = 0.0;
  for (int j = -rh; j <= rh; j++) {
    const bool edge_y = j == -rh || j == rh;
    for (int i = -rw; i <= rw; i++)
      if (!(edge_y && (i == -rw || i == rw))) mean += (double)img[(size_t)(y + j) * W + x + i];
  }
  mean /= (double)patch_size;
  // :143-171: mean-subtract and min/max over the ellipse (raster order).
  double mn = DBL_MAX, mx = -DBL_MAX;
  for (int k = 0; k < e.k; k++) {
    const double p = (double)img[(size_t)(y + e.dy[k]) * W + x + e.dx[k]] - mean;
    mn = p < mn ? p : mn;
    mx = mx < p ? p : mx;
  }
  const double den = mx - mn + (double)kEps;
  // every element is divided by the block's one divisor: its correctly
  // rounded reciprocal once, then Markstein's correction per element (the
  // IEEE quotient, for three FP64 operations instead of a division)
  const double rden = __drcp_rn(den);
  // :174-205: remap to [0, 1] and raw moments (1-based coordinates).
  double m00 = 0.0, m10 = 0.0, m01 = 0.0;
  for (int k = 0; k < e.k; k++) {
    const double r = div_fixed(((double)img[(size_t)(y + e.dy[k]) * W + x + e.dx[k]] - mean) - mn, den, rden);
    m00 += r;
    m10 += (double)(e.dx[k] + rw + 1) * r;
    m01 += (double)(e.dy[k] + rh + 1) * r;
  }
  // :207-239: central moments around that centroid with 0-based coordinates.
  const double cx = m10 / (m00 + (double)kEps), cy = m01 / (m00 + (double)kEps);
  double mu20 = 0.0, mu02 = 0.0;
  for (int k = 0; k < e.k; k++) {
    const double r = div_fixed(((double)img[(size_t)(y + e.dy[k]) * W + x + e.dx[k]] - mean) - mn, den, rden);
    const double ax = (double)(e.dx[k] + rw) - cx, ay = (double)(e.dy[k] + rh) - cy;
    mu20 += (ax * ax) * r;
    mu02 += (ay * ay) * r;
  }
  const double m2 = m00 * m00 + (double)kEps;
  const double hu1 = mu20 / m2 + mu02 / m2;
  out[idx] = (float)sqrt(ref_hu1 * hu1);  // :267
}

// ---------------------------------------------------------------------------
// Block-map Hu distance: the seven Hu invariants of each block against the
// reference block's, one thread per pixel (FP64; hu7_invariants).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_block_hu7(const float* __restrict__ img_all, int W, int H, Ellipse e, Hu7Ref ref, float* __restrict__ out_all,
                float* __restrict__ stds_out) {
  const size_t plane = (size_t)W * H;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= plane) return;
  const size_t off = (size_t)blockIdx.y * plane;
  const float* img = img_all + off;
  const int x = (int)(idx % W), y = (int)(idx / W);
  if (x < e.rw || x >= W - e.rw || y < e.rh || y >= H - e.rh) {
    out_all[off + idx] = 0.0f;
    if (stds_out) stds_out[off + idx] = 0.0f;
    return;
  }
  const float* c = img + idx;
  if (stds_out) {
    float m, sd;
    block_stats_f32(c, W, e, &m, &sd);
    stds_out[off + idx] = sd;
  }
  double h[7];
  hu7_invariants([&](int k) { return (double)__ldg(c + e.dy[k] * W + e.dx[k]); }, e, h);
  out_all[off + idx] = (float)hu7_distance(h, ref.h);
}

void launch_block_hu7(const float* img, int W, int H, int frames, const Ellipse& e, const Hu7Ref& ref, float* out,
                      float* stds_out, cudaStream_t st) {
  const size_t plane = (size_t)W * H;
  k_block_hu7<<<dim3((unsigned)((plane + 127) / 128), (unsigned)frames), 128, 0, st>>>(img, W, H, e, ref, out,
                                                                                        stds_out);
}

void hu7_reference(const float* ref_pixels, const Ellipse& e, Hu7Ref* out) {
  hu7_invariants([&](int k) { return (double)ref_pixels[k]; }, e, out->h);
}

// ---------------------------------------------------------------------------
// Hu map, kernelGetHuMap.cl (FP32): per-block feature, then all pairs.
// ---------------------------------------------------------------------------

// :62-80 / :109-124 with getInvariant (:146-172): the whole square block minus
// the block's local mean; invariant(2,0) + invariant(0,2). Both invariants
// accumulate mu_00 in the same order, so it is summed once.
__global__ void k_hu_features(const float* __restrict__ img, const float* __restrict__ means,
                              const float* __restrict__ stds, int W, int bw, int bh, int nx, int n,
                              float* __restrict__ feat, float* __restrict__ sig) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int rw = bw / 2, rh = bh / 2;
  const int x = rw + t % nx, y = rh + t / nx;
  float x_avg = 0.0f;
  for (int i = 1; i <= bw; i++) x_avg += (float)i;
  x_avg /= (float)bw;
  float y_avg = 0.0f;
  for (int i = 1; i <= bh; i++) y_avg += (float)i;
  y_avg /= (float)bh;
  const float m = means[(size_t)y * W + x];
  float s20 = 0.0f, s02 = 0.0f, m00 = 0.0f;
  for (int j = 0; j < bh; j++) {
    const float b = (float)j + 1.0f - y_avg;
    for (int i = 0; i < bw; i++) {
      const float a = (float)i + 1.0f - x_avg;
      const float p = img[(size_t)(y - rh + j) * W + x - rw + i] - m;
      s20 += (a * a) * p;  // pow(a, 2) * pow(b, 0) * p
      s02 += (b * b) * p;  // pow(a, 0) * pow(b, 2) * p
      m00 += p;
    }
  }
  const float mu00 = m00 * m00;  // pow(mu_00, 1 + (p + q) / 2) with p + q = 2
  feat[t] = s20 / (mu00 + kEps) + s02 / (mu00 + kEps);
  sig[t] = stds[(size_t)y * W + x];
}

constexpr int kHuChunk = 2048;

// :82-132: hu_map[p] = sum_q |hu_q - hu_p| * weight(sigma_p, sigma_q), with
// weight = (100^similarity - 1) / 99 (getExpDecayWeight, :136-144). One
// thread per reference block; FP32 terms, FP32 runs of 32 added into FP64.
__global__ void __launch_bounds__(256)
    k_hu_pairs(const float* __restrict__ feat, const float* __restrict__ sig, int n, int W, int rw, int rh,
               int nx, float* __restrict__ out) {
  __shared__ float sf[kHuChunk], ss[kHuChunk];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const float hp = p < n ? feat[p] : 0.0f, sp = p < n ? sig[p] : 0.0f;
  const float asp = fabsf(sp);
  double acc = 0.0;
  for (int q0 = 0; q0 < n; q0 += kHuChunk) {
    const int m = min(kHuChunk, n - q0);
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      sf[i] = feat[q0 + i];
      ss[i] = sig[q0 + i];
    }
    __syncthreads();
    for (int t0 = 0; t0 < m; t0 += 32) {
      const int t1 = min(m, t0 + 32);
      float part = 0.0f;
      for (int t = t0; t < t1; t++) {
        const float sq = ss[t];
        const float sim = 1.0f - __fdiv_rn(fabsf(sp - sq), asp + fabsf(sq) + kEps);
        const float w = __fdiv_rn(exp2f(sim * kLog2Hundred) - 1.0f, 99.0f);
        part += fabsf(sf[t] - hp) * w;
      }
      acc += (double)part;
    }
  }
  if (p < n) out[(size_t)(rh + p / nx) * W + rw + p % nx] = (float)acc;
}

// ---------------------------------------------------------------------------
// Phase correlation (kernelGetPhaseCorrelationMap.cl with its three defects
// repaired), FP64.
// ---------------------------------------------------------------------------

// Twiddles of both axes into shared memory, all threads of the block.
__device__ __forceinline__ void phase_twiddles_smem(int bw, int bh, double* cw, double* sw, double* ch,
                                                    double* sh) {
  for (int t = threadIdx.x; t < bw * bw; t += blockDim.x) {
    const double ang = 2 * kPhasePi * (1.0 * (t / bw) * (t % bw) / bw);
    cw[t] = cos(ang);
    sw[t] = sin(ang);
  }
  for (int t = threadIdx.x; t < bh * bh; t += blockDim.x) {
    const double ang = 2 * kPhasePi * (1.0 * (t / bh) * (t % bh) / bh);
    ch[t] = cos(ang);
    sh[t] = sin(ang);
  }
}

// :46-71 / :80-106: DFT of every interior block's whole square patch,
// normalised as (x - mean) / (std + eps). F[q * bw*bh + k].
__global__ void __launch_bounds__(128)
    k_phase_dft(const float* __restrict__ img, const float* __restrict__ means, const float* __restrict__ stds,
                int W, int bw, int bh, int nx, int n, double* __restrict__ fr, double* __restrict__ fi) {
  __shared__ double tw[4 * kPhaseMaxN];
  double *cw = tw, *sw = tw + bw * bw, *ch = sw + bw * bw, *sh = ch + bh * bh;
  phase_twiddles_smem(bw, bh, cw, sw, ch, sh);
  __syncthreads();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int rw = bw / 2, rh = bh / 2, nn = bw * bh;
  const int x = rw + q % nx, y = rh + q / nx;
  const double m = (double)means[(size_t)y * W + x], s = (double)stds[(size_t)y * W + x] + (double)kEps;
  double work[kPhaseMaxN + kPhaseTmp];  // [patch | temporaries]
  double* xg = work;
  for (int j = 0; j < bh; j++)
    for (int i = 0; i < bw; i++) xg[j * bw + i] = ((double)img[(size_t)(y - rh + j) * W + x - rw + i] - m) / s;
  phase_dft(xg, bw, bh, cw, sw, ch, sh, fr + (size_t)q * nn, fi + (size_t)q * nn, work + kPhaseMaxN);
}

// Block-map form: the reference block's DFT against each block's. Blocks are
// normalised with their FP32 local statistics (computed here, and written to
// stds_out when it is given) and restricted to the ellipse (0 elsewhere on
// the bw x bh grid).
//
// A group of D = max(bw, bh) lanes evaluates one pixel at a time: a warp
// holds P = 32 / D groups, a CTA 4P, and each group takes D consecutive
// pixels in turn (lane t computes the local statistics of the group's pixel t
// up front). The separable transforms run one line per lane: the lane holds
// its line (a patch row, a half-transformed column, ...) in registers and
// walks the outputs, so the twiddles are the only operands it loads, and
// every lane of the warp loads the same one (a broadcast). Between stages the
// lines go through the group's two shared buffers (real, imaginary).
// Every output is the same sequential sum as in phase_dft (forward) and in the
// kernel's inverse DFT (:132-142: rows over ii, then columns over jj), and the
// peak search keeps the kernel's rule (:144-157: the largest value above 0,
// the lowest raster index on ties), so the map equals the one-thread-per-pixel
// evaluation of the oracle.
// Pixels outside the interior (and past the plane) run on a zero patch and
// are written as 0, so the warp stays converged for its shuffles.
template <int D>
struct PhaseShape {
  static constexpr int P = 32 / D;       // groups per warp
  static constexpr int NG = 4 * P;       // groups per CTA
  static constexpr int PIX = NG * D;     // pixels per CTA
};

// Inverse DFT (real part) of the cross-power spectrum X held in a group's
// buffers (X(j, i) at j * bw + i; overwritten) and its peak: each lane of the
// group (t < D; t = D takes no line) holds one line in registers, as in the
// forward transform, and every output keeps the kernel's sequential sums
// (:132-142: S(i, jj) over ii, then v(j, i) over jj, divided by sqrt(bw bh)).
// Returns, in the group's lane t = 0, the raster index of the
// largest value above 0 (lowest index on ties), -1 if none. All 32 lanes of
// the warp call it together; lr and li are the caller's line registers.
template <int D>
__device__ __forceinline__ int phase_group_peak(double* re, double* im, const double* cw, const double* sw,
                                                const double* ch, const double* sh, int bw, int bh, double sn,
                                                int t, double (&lr)[D], double (&li)[D]) {
  const unsigned full = 0xffffffffu;
  // inverse, rows: lane jj holds X(jj, :); S(i, jj) = sum_ii X[jj][ii] e^{+i a(i, ii)}
  if (t < bh) {
#pragma unroll
    for (int ii = 0; ii < D; ii++) {
      lr[ii] = ii < bw ? re[t * bw + ii] : 0.0;
      li[ii] = ii < bw ? im[t * bw + ii] : 0.0;
    }
  }
  __syncwarp();
  if (t < bh) {
    for (int i = 0; i < bw; i++) {
      double sr = 0.0, si = 0.0;
#pragma unroll
      for (int ii = 0; ii < D; ii++) {
        if (ii < bw) {
          const double c = cw[i * bw + ii], s = sw[i * bw + ii];
          sr += lr[ii] * c - li[ii] * s;
          si += lr[ii] * s + li[ii] * c;
        }
      }
      re[i * bh + t] = sr;
      im[i * bh + t] = si;
    }
  }
  __syncwarp();
  // inverse, columns (real part): lane i holds S(i, :);
  // v(j, i) = sum_jj Re(S(i, jj) e^{+i b(j, jj)}) / sn, and the lane's peak
  double best = 0.0;
  int bidx = -1;
  if (t < bw) {
#pragma unroll
    for (int jj = 0; jj < D; jj++) {
      lr[jj] = jj < bh ? re[t * bh + jj] : 0.0;
      li[jj] = jj < bh ? im[t * bh + jj] : 0.0;
    }
    for (int j = 0; j < bh; j++) {
      double v = 0.0;
#pragma unroll
      for (int jj = 0; jj < D; jj++)
        if (jj < bh) v += lr[jj] * ch[j * bh + jj] - li[jj] * sh[j * bh + jj];
      v /= sn;
      const int k = j * bw + t;
      if (v > best || (bidx >= 0 && v == best && k < bidx)) {
        best = v;
        bidx = k;
      }
    }
  }
  // the group's peak (lane t gathers lanes t .. t + 2o - 1 of the group):
  // largest value above 0, lowest raster index on ties
#pragma unroll
  for (int o = 1; o < D; o <<= 1) {
    const double ob = __shfl_down_sync(full, best, o);
    const int oi = __shfl_down_sync(full, bidx, o);
    if (t + o < D && oi >= 0 && (bidx < 0 || ob > best || (ob == best && oi < bidx))) {
      best = ob;
      bidx = oi;
    }
  }
  return bidx;
}

// Block-map form (this library's definition; the reference wires phase
// correlation into no block map): the exact DFT, twiddles e^{-2 pi i m / L}
// (PhaseRef), of each block normalised as (x - mean) / (std + eps) with its FP32
// local statistics and restricted to the ellipse, the kernel's normalised
// cross-power spectrum with the reference block's DFT, the real part of the
// inverse DFT and the kernel's peak rule (largest value above 0, lowest raster
// index on ties; 1-based coordinates). With exact roots of unity a length-L
// line transform pairs x_n with x_{L-n}: a_n = x_n + x_{L-n} and
// b_n = x_n - x_{L-n} share the cosine and sine of each output pair (k, L - k),
// (L - 1)^2 real multiply-adds per complex line instead of 4 L^2, and the
// forward transform of the real patch is Hermitian, so it needs half its rows'
// outputs and (bw + 1) / 2 column lines. Lines are read from the group's
// shared buffers already paired, so every register index is a compile-time
// constant.
//
// A group of D = max(bw, bh) lanes evaluates one pixel at a time as in the
// all-pairs kernel (PhaseShape): lane t holds line t of each stage.
// phase_cross with x / sn given as x and 1/sn, and the two quotients by the
// shared denominator as one correctly rounded reciprocal and Markstein's
// correction (div_fixed): every quotient is the IEEE one, as in phase_cross.
__device__ __forceinline__ void phase_cross_fixed(double rr, double ri, double fr, double fi, double sn, double rsn,
                                                  double* xr, double* xi) {
  const double qr = div_fixed(fr, sn, rsn), qi = div_fixed(fi, sn, rsn);
  const double conj = (-1) * qi;
  const double mr = rr * qr - ri * conj;
  const double mi = rr * conj + ri * qr;
  const double ar = fabs(mr), ai = fabs(mi);
  const double den = (ar * ar) + (ai * ai) + (double)kEps;
  const double rden = __drcp_rn(den);
  *xr = div_fixed((mr * ar) + (mi * ai), den, rden);
  *xi = div_fixed((mi * ar) - (mr * ai), den, rden);
}

template <int D>
__global__ void __launch_bounds__(128)
    k_block_phase(const float* __restrict__ img_all, int W, int H, Ellipse e, int bw, int bh, PhaseRef ref,
                  float* __restrict__ out_all, float* __restrict__ stds_out) {
  using S = PhaseShape<D>;
  constexpr int HD = (D - 1) / 2;
  __shared__ double tcw[HD * HD + 1], tsw[HD * HD + 1], tch[HD * HD + 1], tsh[HD * HD + 1];
  __shared__ double rre[D * D], rim[D * D];
  __shared__ double buf[S::NG][2 * D * D];
  __shared__ int s_img[D * D], s_grid[D * D];  // ellipse: image offset, patch position
  const int hw = (bw - 1) / 2, hh = (bh - 1) / 2;
  // c(n, k) = cos(2 pi (n k mod L) / L) at (n - 1) HD + k - 1, n, k = 1 .. (L - 1) / 2
  for (int k = threadIdx.x; k < HD * HD; k += blockDim.x) {
    const int n = k / HD + 1, m = k % HD + 1;
    tcw[k] = n <= hw && m <= hw ? ref.cw[(n * m) % bw] : 0.0;
    tsw[k] = n <= hw && m <= hw ? ref.sw[(n * m) % bw] : 0.0;
    tch[k] = n <= hh && m <= hh ? ref.ch[(n * m) % bh] : 0.0;
    tsh[k] = n <= hh && m <= hh ? ref.sh[(n * m) % bh] : 0.0;
  }
  const int nn = bw * bh;
  for (int k = threadIdx.x; k < nn; k += blockDim.x) {
    rre[k] = ref.re[k];
    rim[k] = ref.im[k];
  }
  for (int k = threadIdx.x; k < e.k; k += blockDim.x) {
    s_img[k] = e.dy[k] * W + e.dx[k];
    s_grid[k] = (e.dy[k] + e.rh) * bw + e.dx[k] + e.rw;
  }
  __syncthreads();
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // lanes past the warp's last group take no line (t = D) and no buffer
  const bool live = lane < S::P * D;
  const int gw = live ? lane / D : 0;
  const int t = live ? lane - gw * D : D;
  const int base = gw * D;  // the group's first lane
  double* re = buf[warp * S::P + gw];
  double* im = re + D * D;
  const size_t plane = (size_t)W * H;
  const size_t off = (size_t)blockIdx.y * plane;
  const float* img = img_all + off;
  float* out = out_all + off;
  const int rw = e.rw, rh = e.rh;
  const double sn = sqrt((double)(bw * bh)), rsn = __drcp_rn(sn);
  const size_t first = (size_t)blockIdx.x * S::PIX + (size_t)(warp * S::P + gw) * D;
  // local statistics of the group's D pixels, lane t for pixel first + t
  float own_m = 0.0f, own_s = 0.0f;
  if (live) {
    const size_t idx = first + t;
    const int x = (int)(idx % W), y = (int)(idx / W);
    if (idx < plane && x >= rw && x < W - rw && y >= rh && y < H - rh) {
      // block_stats_f32's sequence over the offsets in shared memory
      const float* c = img + idx;
      float sum = 0.0f;
      for (int i = 0; i < e.k; i++) sum = __fadd_rn(sum, c[s_img[i]]);
      own_m = __fdiv_rn(sum, (float)e.k);
      float v = 0.0f;
      for (int i = 0; i < e.k; i++) {
        const float d = __fsub_rn(c[s_img[i]], own_m);
        v = __fadd_rn(v, __fmul_rn(d, d));
      }
      own_s = __fsqrt_rn(__fdiv_rn(v, (float)(e.k - 1)));
    }
    if (stds_out && idx < plane) stds_out[off + idx] = own_s;
  }
  for (int n = 0; n < D; n++) {
    const size_t idx = first + n;
    const int x = (int)(idx % W), y = (int)(idx / W);
    const bool act = idx < plane && x >= rw && x < W - rw && y >= rh && y < H - rh;
    const float mf = __shfl_sync(full, own_m, base + n);
    const float sf = __shfl_sync(full, own_s, base + n);
    const double m = (double)mf, sd = (double)sf + (double)kEps, rsd = __drcp_rn(sd);
    // the patch, in the real buffer
    if (live)
      for (int k = t; k < nn; k += D) re[k] = 0.0;
    __syncwarp();
    if (live && act) {
      const float* c = img + (size_t)y * W + x;
      for (int k = t; k < e.k; k += D) re[s_grid[k]] = div_fixed((double)c[s_img[k]] - m, sd, rsd);
    }
    __syncwarp();
    // paired line registers: x0, a_n, b_n (n = 1 .. HD), real and imaginary
    double x0r = 0.0, x0i = 0.0, ar[HD], ai[HD], br[HD], bi[HD];
    // forward, rows (real): lane jj, T(i, jj) for i = 0 .. hw
    if (t < bh) {
      const double* row = re + t * bw;
      x0r = row[0];
#pragma unroll
      for (int q = 1; q <= HD; q++) {
        const double u = q <= hw ? row[q] : 0.0, v = q <= hw ? row[bw - q] : 0.0;
        ar[q - 1] = u + v;
        br[q - 1] = u - v;
      }
    }
    __syncwarp();
    if (t < bh) {
      double s0 = x0r;
#pragma unroll
      for (int q = 0; q < HD; q++) s0 += ar[q];
      re[t] = s0;  // T(0, jj) at 0 * bh + jj
      im[t] = 0.0;
      for (int k = 1; k <= hw; k++) {
        double pr = x0r, qi = 0.0;
#pragma unroll
        for (int q = 0; q < HD; q++) {
          pr = __fma_rn(ar[q], tcw[q * HD + k - 1], pr);
          qi = __fma_rn(br[q], tsw[q * HD + k - 1], qi);
        }
        re[k * bh + t] = pr;  // e^{-i}: X_k = P - i Q
        im[k * bh + t] = -qi;
      }
    }
    __syncwarp();
    // forward, columns i = 0 .. hw (complex): F(j, i); the mirrored columns
    // bw - i are F(bh - j, bw - i) = conj(F(j, i)). Each output leaves as the
    // normalised cross-power spectrum X with the reference.
    if (t <= hw) {
      const double* cr = re + t * bh;
      const double* ci = im + t * bh;
      x0r = cr[0];
      x0i = ci[0];
#pragma unroll
      for (int q = 1; q <= HD; q++) {
        const bool in = q <= hh;
        const double ur = in ? cr[q] : 0.0, ui = in ? ci[q] : 0.0;
        const double vr = in ? cr[bh - q] : 0.0, vi = in ? ci[bh - q] : 0.0;
        ar[q - 1] = ur + vr;
        ai[q - 1] = ui + vi;
        br[q - 1] = ur - vr;
        bi[q - 1] = ui - vi;
      }
    }
    __syncwarp();
    if (t <= hw) {
      auto emit = [&](int j, double fr, double fi) {
        const int k = j * bw + t;
        phase_cross_fixed(rre[k], rim[k], fr, fi, sn, rsn, &re[k], &im[k]);
        if (t > 0) {  // the mirrored column: conj(F(j, t)) at (bh - j) mod bh, bw - t
          const int k2 = ((bh - j) % bh) * bw + bw - t;
          phase_cross_fixed(rre[k2], rim[k2], fr, -fi, sn, rsn, &re[k2], &im[k2]);
        }
      };
      double s0r = x0r, s0i = x0i;
#pragma unroll
      for (int q = 0; q < HD; q++) {
        s0r += ar[q];
        s0i += ai[q];
      }
      emit(0, s0r, s0i);
      for (int k = 1; k <= hh; k++) {
        double prr = x0r, pri = x0i, qr = 0.0, qi = 0.0;
#pragma unroll
        for (int q = 0; q < HD; q++) {
          const double c = tch[q * HD + k - 1], s = tsh[q * HD + k - 1];
          prr = __fma_rn(ar[q], c, prr);
          pri = __fma_rn(ai[q], c, pri);
          qr = __fma_rn(br[q], s, qr);
          qi = __fma_rn(bi[q], s, qi);
        }
        emit(k, prr + qi, pri - qr);       // P - i Q
        emit(bh - k, prr - qi, pri + qr);  // P + i Q
      }
    }
    __syncwarp();
    // inverse, rows (complex): lane jj holds X(jj, :); S(i, jj) = sum_ii X(jj, ii) e^{+i a(i, ii)}
    if (t < bh) {
      const double* xr = re + t * bw;
      const double* xi = im + t * bw;
      x0r = xr[0];
      x0i = xi[0];
#pragma unroll
      for (int q = 1; q <= HD; q++) {
        const bool in = q <= hw;
        const double ur = in ? xr[q] : 0.0, ui = in ? xi[q] : 0.0;
        const double vr = in ? xr[bw - q] : 0.0, vi = in ? xi[bw - q] : 0.0;
        ar[q - 1] = ur + vr;
        ai[q - 1] = ui + vi;
        br[q - 1] = ur - vr;
        bi[q - 1] = ui - vi;
      }
    }
    __syncwarp();
    if (t < bh) {
      double s0r = x0r, s0i = x0i;
#pragma unroll
      for (int q = 0; q < HD; q++) {
        s0r += ar[q];
        s0i += ai[q];
      }
      re[t] = s0r;
      im[t] = s0i;
      for (int k = 1; k <= hw; k++) {
        double prr = x0r, pri = x0i, qr = 0.0, qi = 0.0;
#pragma unroll
        for (int q = 0; q < HD; q++) {
          const double c = tcw[q * HD + k - 1], s = tsw[q * HD + k - 1];
          prr = __fma_rn(ar[q], c, prr);
          pri = __fma_rn(ai[q], c, pri);
          qr = __fma_rn(br[q], s, qr);
          qi = __fma_rn(bi[q], s, qi);
        }
        re[k * bh + t] = prr - qi;  // P + i Q
        im[k * bh + t] = pri + qr;
        re[(bw - k) * bh + t] = prr + qi;  // P - i Q
        im[(bw - k) * bh + t] = pri - qr;
      }
    }
    __syncwarp();
    // inverse, columns (real part): lane i holds S(i, :); v(j, i) = Re sum_jj S(i, jj) e^{+i b(j, jj)} / sn
    double best = 0.0;
    int bidx = -1;
    if (t < bw) {
      const double* cr = re + t * bh;
      const double* ci = im + t * bh;
      x0r = cr[0];
#pragma unroll
      for (int q = 1; q <= HD; q++) {
        const bool in = q <= hh;
        const double ur = in ? cr[q] : 0.0, ui = in ? ci[q] : 0.0;
        const double vr = in ? cr[bh - q] : 0.0, vi = in ? ci[bh - q] : 0.0;
        ar[q - 1] = ur + vr;  // real parts of a_n
        bi[q - 1] = ui - vi;  // imaginary parts of b_n
      }
      auto cand = [&](int j, double v) {
        v = div_fixed(v, sn, rsn);
        const int k = j * bw + t;
        if (v > best || (bidx >= 0 && v == best && k < bidx)) {
          best = v;
          bidx = k;
        }
      };
      double s0 = x0r;
#pragma unroll
      for (int q = 0; q < HD; q++) s0 += ar[q];
      cand(0, s0);
      for (int k = 1; k <= hh; k++) {
        double pr = x0r, qi = 0.0;
#pragma unroll
        for (int q = 0; q < HD; q++) {
          pr = __fma_rn(ar[q], tch[q * HD + k - 1], pr);
          qi = __fma_rn(bi[q], tsh[q * HD + k - 1], qi);
        }
        cand(k, pr - qi);       // Re(P + i Q)
        cand(bh - k, pr + qi);  // Re(P - i Q)
      }
    }
    // the group's peak (lane t gathers lanes t .. t + 2o - 1 of the group):
    // largest value above 0, lowest raster index on ties
#pragma unroll
    for (int o = 1; o < D; o <<= 1) {
      const double ob = __shfl_down_sync(full, best, o);
      const int oi = __shfl_down_sync(full, bidx, o);
      if (t + o < D && oi >= 0 && (bidx < 0 || ob > best || (ob == best && oi < bidx))) {
        best = ob;
        bidx = oi;
      }
    }
    if (t == 0 && idx < plane) {
      float r = 0.0f;
      if (act && bidx >= 0) {
        const double px = (double)(bidx % bw + 1), py = (double)(bidx / bw + 1);
        r = (float)sqrt((px * px) + (py * py));
      }
      out[idx] = r;
    }
    __syncwarp();
  }
}

template <int D>
void launch_block_phase_t(const float* img, int W, int H, int frames, const Ellipse& e, int bw, int bh,
                          const PhaseRef& ref, float* out, float* stds_out, cudaStream_t st) {
  const dim3 grid((unsigned)(((size_t)W * H + PhaseShape<D>::PIX - 1) / PhaseShape<D>::PIX), (unsigned)frames);
  k_block_phase<D><<<grid, 128, 0, st>>>(img, W, H, e, bw, bh, ref, out, stds_out);
}

void launch_block_phase(const float* img, int W, int H, int frames, const Ellipse& e, int bw, int bh,
                        const PhaseRef& ref, float* out, float* stds_out, cudaStream_t st) {
  const int d = bw > bh ? bw : bh;
  if (d <= 3)
    launch_block_phase_t<3>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
  else if (d <= 5)
    launch_block_phase_t<5>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
  else if (d <= 7)
    launch_block_phase_t<7>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
  else if (d <= 9)
    launch_block_phase_t<9>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
  else if (d <= 11)
    launch_block_phase_t<11>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
  else if (d <= 13)
    launch_block_phase_t<13>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
  else
    launch_block_phase_t<15>(img, W, H, frames, e, bw, bh, ref, out, stds_out, st);
}

// :73-163: one CTA per reference block p; phase_map[p] = sum_q |peak_pq| *
// weight(sigma_p, sigma_q). The CTA's groups of D lanes (PhaseShape) take the
// comparison blocks q in turn: the cross-power spectrum of the two stored DFTs
// spread over the group's lanes, then phase_group_peak. Each group sums its
// pairs in FP64 in q order, and the CTA adds the groups' sums in group order.
template <int D>
__global__ void __launch_bounds__(128)
    k_phase_pairs(const double* __restrict__ fr, const double* __restrict__ fi, const float* __restrict__ sig,
                  int n, int bw, int bh, int W, int nx, float* __restrict__ out) {
  using S = PhaseShape<D>;
  __shared__ double tw[4 * D * D];
  __shared__ double pr[D * D], pi[D * D];
  __shared__ double buf[S::NG][2 * D * D];
  __shared__ double red[S::NG];
  double *cw = tw, *sw = tw + bw * bw, *ch = sw + bw * bw, *sh = ch + bh * bh;
  const int p = blockIdx.x, nn = bw * bh;
  phase_twiddles_smem(bw, bh, cw, sw, ch, sh);
  for (int k = threadIdx.x; k < nn; k += blockDim.x) {
    pr[k] = fr[(size_t)p * nn + k];
    pi[k] = fi[(size_t)p * nn + k];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool live = lane < S::P * D;  // lanes past the warp's last group take no line
  const int gw = live ? lane / D : 0;
  const int t = live ? lane - gw * D : D;
  const int g = warp * S::P + gw;
  double* re = buf[g];
  double* im = re + D * D;
  const float sp = sig[p];
  const double sn = sqrt((double)(bw * bh));
  double acc = 0.0;  // the group's sum, in its lane t = 0
  // every group of a warp runs the same rounds, so the warp stays converged
  const int rounds = (n + S::NG - 1) / S::NG;
  for (int r = 0; r < rounds; r++) {
    const int q = r * S::NG + g;
    const bool act = live && q < n;
    if (act) {
      const double* qr = fr + (size_t)q * nn;
      const double* qi = fi + (size_t)q * nn;
      for (int k = t; k < nn; k += D) phase_cross(pr[k], pi[k], qr[k], qi[k], &re[k], &im[k]);
    }
    __syncwarp();
    double lr[D], li[D];
    const int bidx = phase_group_peak<D>(re, im, cw, sw, ch, sh, bw, bh, sn, act ? t : D, lr, li);
    if (act && t == 0) {
      float d = 0.0f;
      if (bidx >= 0) {
        const double px = (double)(bidx % bw + 1), py = (double)(bidx / bw + 1);
        d = (float)sqrt((px * px) + (py * py));
      }
      acc += (double)d * (double)phase_weight(sp, sig[q]);
    }
    __syncwarp();
  }
  if (live && t == 0) red[g] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int i = 0; i < S::NG; i++) sum += red[i];
    const int rw = bw / 2, rh = bh / 2;
    out[(size_t)(rh + p / nx) * W + rw + p % nx] = (float)sum;
  }
}

template <int D>
void launch_phase_pairs_t(const double* fr, const double* fi, const float* sig, int n, int bw, int bh, int W, int nx,
                          float* out, cudaStream_t st) {
  k_phase_pairs<D><<<n, 128, 0, st>>>(fr, fi, sig, n, bw, bh, W, nx, out);
}

void launch_phase_pairs(const double* fr, const double* fi, const float* sig, int n, int bw, int bh, int W, int nx,
                        float* out, cudaStream_t st) {
  const int d = bw > bh ? bw : bh;
  if (d <= 3)
    launch_phase_pairs_t<3>(fr, fi, sig, n, bw, bh, W, nx, out, st);
  else if (d <= 5)
    launch_phase_pairs_t<5>(fr, fi, sig, n, bw, bh, W, nx, out, st);
  else if (d <= 7)
    launch_phase_pairs_t<7>(fr, fi, sig, n, bw, bh, W, nx, out, st);
  else if (d <= 9)
    launch_phase_pairs_t<9>(fr, fi, sig, n, bw, bh, W, nx, out, st);
  else if (d <= 11)
    launch_phase_pairs_t<11>(fr, fi, sig, n, bw, bh, W, nx, out, st);
  else if (d <= 13)
    launch_phase_pairs_t<13>(fr, fi, sig, n, bw, bh, W, nx, out, st);
  else
    launch_phase_pairs_t<15>(fr, fi, sig, n, bw, bh, W, nx, out, st);
}

// Values of `a` at the interior pixels, in interior raster order.
__global__ void k_gather_interior(const float* __restrict__ a, int W, int rw, int rh, int nx, int n,
                                  float* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = a[(size_t)(rh + t / nx) * W + rw + t % nx];
}

// ---------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------

// The reference block of the block-map Hu metric: ReferenceBlock2D pixels
// (ellipse order) on the bw x bh grid, mean-subtracted over the ellipse and
// min-max remapped to [0, 1] in FP64 as kernelGetPatchHu2D.cl:126-182 does to
// every comparison patch; stored as float like the kernel's patch buffer.
void hu_prepare_patch(const float* ref_pixels, int bw, int bh, float* grid) {
  Ellipse e;
  const int K = build_ellipse(bw, bh, &e);
  double v[kMaxK];
  double mean = 0.0;
  for (int k = 0; k < K; k++) {
    v[k] = (double)ref_pixels[k];
    mean += v[k];
  }
  mean /= (double)K;
  double mn = DBL_MAX, mx = -DBL_MAX;
  for (int k = 0; k < K; k++) {
    v[k] -= mean;
    mn = v[k] < mn ? v[k] : mn;
    mx = mx < v[k] ? v[k] : mx;
  }
  for (int i = 0; i < bw * bh; i++) grid[i] = 0.0f;
  for (int k = 0; k < K; k++)
    grid[(e.dy[k] + e.rh) * bw + e.dx[k] + e.rw] = (float)((v[k] - mn) / (mx - mn + (double)kEps));
}

// Hu invariant 1 of the patch as kernelGetPatchHu2D.cl:51-101 computes it for
// its reference patch.
double patch_hu1(const float* patch, int bw, int bh) {
  Ellipse e;
  const int K = build_ellipse(bw, bh, &e);
  double m00 = 0.0, m10 = 0.0, m01 = 0.0;
  for (int k = 0; k < K; k++) {
    const int i = e.dx[k] + e.rw, j = e.dy[k] + e.rh;
    const double p = (double)patch[j * bw + i];
    m00 += p;
    m10 += (double)(i + 1) * p;
    m01 += (double)(j + 1) * p;
  }
  const double cx = m10 / (m00 + (double)kEps), cy = m01 / (m00 + (double)kEps);
  double mu20 = 0.0, mu02 = 0.0;
  for (int k = 0; k < K; k++) {
    const int i = e.dx[k] + e.rw, j = e.dy[k] + e.rh;
    const double p = (double)patch[j * bw + i];
    mu20 += pow(((double)i - cx), 2.0) * p;
    mu02 += pow(((double)j - cy), 2.0) * p;
  }
  const double nu20 = mu20 / (pow(m00, 2.0) + (double)kEps);
  const double nu02 = mu02 / (pow(m00, 2.0) + (double)kEps);
  return nu20 + nu02;
}

void phase_reference_dft(const float* ref_pixels, float ref_std, int bw, int bh, PhaseRef* out) {
  Ellipse e;
  const int K = build_ellipse(bw, bh, &e);
  const double two_pi = 6.283185307179586476925286766559;
  for (int m = 0; m < bw; m++) {
    out->cw[m] = std::cos(two_pi * m / bw);
    out->sw[m] = std::sin(two_pi * m / bw);
  }
  for (int m = 0; m < bh; m++) {
    out->ch[m] = std::cos(two_pi * m / bh);
    out->sh[m] = std::sin(two_pi * m / bh);
  }
  double xg[kPhaseMaxN], tr[kPhaseMaxN], ti[kPhaseMaxN];
  for (int k = 0; k < bw * bh; k++) xg[k] = 0.0;
  for (int k = 0; k < K; k++)
    xg[(e.dy[k] + e.rh) * bw + e.dx[k] + e.rw] = (double)ref_pixels[k] / ((double)ref_std + (double)kEps);
  // exact DFT, direct sums: rows, then columns
  for (int jj = 0; jj < bh; jj++)
    for (int i = 0; i < bw; i++) {
      double sr = 0.0, si = 0.0;
      for (int ii = 0; ii < bw; ii++) {
        const int m = (i * ii) % bw;
        sr += xg[jj * bw + ii] * out->cw[m];
        si -= xg[jj * bw + ii] * out->sw[m];
      }
      tr[jj * bw + i] = sr;
      ti[jj * bw + i] = si;
    }
  for (int j = 0; j < bh; j++)
    for (int i = 0; i < bw; i++) {
      double sr = 0.0, si = 0.0;
      for (int jj = 0; jj < bh; jj++) {
        const int m = (j * jj) % bh;
        sr += tr[jj * bw + i] * out->ch[m] + ti[jj * bw + i] * out->sh[m];
        si += ti[jj * bw + i] * out->ch[m] - tr[jj * bw + i] * out->sh[m];
      }
      out->re[j * bw + i] = sr;
      out->im[j * bw + i] = si;
    }
}

}  // namespace sred
