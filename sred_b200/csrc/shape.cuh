// Shape metrics: Hu moments and phase correlation (device and host helpers).
//
// The reference ships three OpenCL kernels for these that its Java code never
// loads (paths relative to src/main/resources/):
//   kernelGetPatchHu2D.cl            one patch against every block, FP64
//   kernelGetHuMap.cl                all pairs of blocks, FP32
//   kernelGetPhaseCorrelationMap.cl  all pairs of blocks, FP64; it does not
//                                    compile as shipped (nUnique undefined,
//                                    :27), its DFT phases divide integers
//                                    (:66, :101, :138) and its peak search
//                                    indexes with the image width (:150).
// libsred evaluates the first two with the kernels' own arithmetic and the
// third with those three defects repaired (no unique-coordinate pre-filter,
// real-valued phases, block-width indexing).
//
// The per-thread work arrays of k_phase_dft live in ONE local array per
// thread, carved into sections by offset. With separate local arrays, a
// one-thread-per-pixel block-map phase kernel built by nvcc 12.9 for sm_100a
// computed DFTs whose first row read overwritten inputs, as if phase_dft's
// column temporaries shared the input patch's stack slots; with one array per
// thread the results were exact. (The block-map and all-pairs kernels now
// keep their lines in registers and shared memory.)
#pragma once
#include <math.h>

#include "common.cuh"

namespace sred {

constexpr int kPhaseMaxDim = 15;                    // phase correlation: bw, bh <= 15
constexpr int kPhaseMaxN = kPhaseMaxDim * kPhaseMaxDim;
constexpr int kPhaseTmp = 2 * kPhaseMaxDim;         // temporaries of phase_dft
// The kernel's pi is a float literal widened to double (:44).
constexpr double kPhasePi = (double)3.14159265358979323846f;
constexpr float kLog2Hundred = 6.64385618977472469574f;  // log2(100)

// Block-map form of phase correlation (exact DFT): the reference block's
// spectrum and the twiddles cos / sin(2 pi m / L) of both axes, m < L,
// computed on the host.
struct PhaseRef {
  double re[kPhaseMaxN];
  double im[kPhaseMaxN];
  double cw[kPhaseMaxDim], sw[kPhaseMaxDim], ch[kPhaseMaxDim], sh[kPhaseMaxDim];
};

// Twiddle tables of one axis: c[a*len+b] = cos(2*PI*(1.0*a*b/len)), s = sin.
// The product a*b is not reduced modulo len: PI is not pi, so the reduction
// would change the angles.
__host__ __device__ inline void phase_twiddles(int len, double* c, double* s) {
  for (int a = 0; a < len; a++)
    for (int b = 0; b < len; b++) {
      const double ang = 2 * kPhasePi * (1.0 * a * b / len);
      c[a * len + b] = cos(ang);
      s[a * len + b] = sin(ang);
    }
}

// F = DFT(x) / sqrt(bw bh) of a real bw x bh patch (x row-major), the
// reference's sum over exp(-i 2 PI (i ii / bw + j jj / bh)) evaluated
// separably one output column at a time:
//   T[jj] = sum_ii x[jj][ii] e^{-i a(i, ii)},  F[j][i] = sum_jj T[jj] e^{-i b(j, jj)}.
// tmp: kPhaseTmp doubles, disjoint from x, fr and fi.
__host__ __device__ inline void phase_dft(const double* x, int bw, int bh, const double* cw, const double* sw,
                                          const double* ch, const double* sh, double* fr, double* fi,
                                          double* tmp) {
  const double sn = sqrt((double)(bw * bh));
  double* tr = tmp;
  double* ti = tmp + kPhaseMaxDim;
  for (int i = 0; i < bw; i++) {
    for (int jj = 0; jj < bh; jj++) {
      double ar = 0.0, ai = 0.0;
      for (int ii = 0; ii < bw; ii++) {
        const double v = x[jj * bw + ii];
        ar += v * cw[i * bw + ii];
        ai -= v * sw[i * bw + ii];
      }
      tr[jj] = ar;
      ti[jj] = ai;
    }
    for (int j = 0; j < bh; j++) {
      double br = 0.0, bi = 0.0;
      for (int jj = 0; jj < bh; jj++) {
        const double c = ch[j * bh + jj], s = sh[j * bh + jj];
        br += tr[jj] * c + ti[jj] * s;
        bi += ti[jj] * c - tr[jj] * s;
      }
      fr[j * bw + i] = br / sn;
      fi[j * bw + i] = bi / sn;
    }
  }
}

// Normalised cross-power of one frequency (:108-130): m = ref * conj(comp),
// out = (m_r|m_r| + m_i|m_i|, m_i|m_r| - m_r|m_i|) / (m_r^2 + m_i^2 + eps).
__host__ __device__ inline void phase_cross(double rr, double ri, double qr, double qi, double* xr, double* xi) {
  const double conj = (-1) * qi;
  const double mr = rr * qr - ri * conj;
  const double mi = rr * conj + ri * qr;
  const double ar = fabs(mr), ai = fabs(mi);
  *xr = ((mr * ar) + (mi * ai)) / ((ar * ar) + (ai * ai) + (double)kEps);
  *xi = ((mi * ar) - (mr * ai)) / ((ar * ar) + (ai * ai) + (double)kEps);
}

// getExpDecayWeight of kernelGetPhaseCorrelationMap.cl:167-179.
__host__ __device__ inline float phase_weight(float ref, float comp) {
  if (ref == comp) return 1.0f;
  return 1 - (2 * (fabsf(ref - comp) / (fabsf(ref) + fabsf(comp))));
}

// Ellipse-block mean and (K-1) standard deviation of the pixel at `c`
// (row stride W) in the FP32 order of cl/kernelGetLocalStatistics2D.cl:15-56,
// the same sequence as k_local_stats.
__device__ __forceinline__ void block_stats_f32(const float* c, int W, const Ellipse& e, float* mean_out,
                                                float* std_out) {
  float s = 0.0f;
  for (int i = 0; i < e.k; i++) s = __fadd_rn(s, c[e.dy[i] * W + e.dx[i]]);
  const float mean = __fdiv_rn(s, (float)e.k);
  float v = 0.0f;
  for (int i = 0; i < e.k; i++) {
    const float d = __fsub_rn(c[e.dy[i] * W + e.dx[i]], mean);
    v = __fadd_rn(v, __fmul_rn(d, d));
  }
  *mean_out = mean;
  *std_out = __fsqrt_rn(__fdiv_rn(v, (float)(e.k - 1)));
}

// Hu's seven moment invariants (M.-K. Hu, "Visual pattern recognition by
// moment invariants", IRE Trans. Inf. Theory 8(2):179-187, 1962) of one
// block's intensities v_k at the ellipse offsets (dx_k, dy_k), in FP64:
// v = (x - min) / (max - min) over the block (every invariant 0 for a flat
// block), centroid from the raw moments, central moments mu_pq for
// p + q = 2, 3, normalised eta_pq = mu_pq / m00^(1 + (p + q) / 2). `get(k)`
// returns x_k as a double; the same function serves the device (image
// blocks) and the host (the reference block), so both sides round alike.
template <class Get>
__host__ __device__ inline void hu7_invariants(Get get, const Ellipse& e, double* h) {
  double mn = get(0), mx = mn;
  for (int k = 1; k < e.k; k++) {
    const double x = get(k);
    mn = x < mn ? x : mn;
    mx = x > mx ? x : mx;
  }
  for (int i = 0; i < 7; i++) h[i] = 0.0;
  const double span = mx - mn;
  if (!(span > 0.0)) return;
  double m00 = 0.0, m10 = 0.0, m01 = 0.0;
  for (int k = 0; k < e.k; k++) {
    const double v = (get(k) - mn) / span;
    m00 += v;
    m10 += (double)e.dx[k] * v;
    m01 += (double)e.dy[k] * v;
  }
  const double cx = m10 / m00, cy = m01 / m00;
  double u20 = 0.0, u11 = 0.0, u02 = 0.0, u30 = 0.0, u21 = 0.0, u12 = 0.0, u03 = 0.0;
  for (int k = 0; k < e.k; k++) {
    const double v = (get(k) - mn) / span;
    const double a = (double)e.dx[k] - cx, b = (double)e.dy[k] - cy;
    const double a2 = a * a, b2 = b * b;
    u20 += a2 * v;
    u11 += (a * b) * v;
    u02 += b2 * v;
    u30 += (a2 * a) * v;
    u21 += (a2 * b) * v;
    u12 += (a * b2) * v;
    u03 += (b2 * b) * v;
  }
  const double s2 = m00 * m00, s3 = s2 * sqrt(m00);
  const double n20 = u20 / s2, n11 = u11 / s2, n02 = u02 / s2;
  const double n30 = u30 / s3, n21 = u21 / s3, n12 = u12 / s3, n03 = u03 / s3;
  const double p = n30 + n12, q = n21 + n03, r = n30 - 3.0 * n12, s = 3.0 * n21 - n03;
  const double d = n20 - n02;
  h[0] = n20 + n02;
  h[1] = d * d + 4.0 * (n11 * n11);
  h[2] = r * r + s * s;
  h[3] = p * p + q * q;
  h[4] = r * p * (p * p - 3.0 * (q * q)) + s * q * (3.0 * (p * p) - q * q);
  h[5] = d * (p * p - q * q) + 4.0 * n11 * p * q;
  h[6] = s * p * (p * p - 3.0 * (q * q)) - r * q * (3.0 * (p * p) - q * q);
}

// L2 distance of two Hu 7-vectors.
__host__ __device__ inline double hu7_distance(const double* a, const double* b) {
  double s = 0.0;
  for (int i = 0; i < 7; i++) {
    const double t = a[i] - b[i];
    s += t * t;
  }
  return sqrt(s);
}

struct Hu7Ref {
  double h[7];
};

// Block-map Hu distance (shape.cu): the frames x W x H raw map (and the FP32
// local stds when stds_out is given) on stream st.
void launch_block_hu7(const float* img, int W, int H, int frames, const Ellipse& e, const Hu7Ref& ref, float* out,
                      float* stds_out, cudaStream_t st);
// The reference block's 7-vector from its ellipse pixels (ReferenceBlock2D).
void hu7_reference(const float* ref_pixels, const Ellipse& e, Hu7Ref* out);

// Block-map phase correlation against the reference block's DFT (shape.cu):
// the frames x W x H raw map (and the FP32 local stds when stds_out is given)
// on stream st; bw, bh <= kPhaseMaxDim.
void launch_block_phase(const float* img, int W, int H, int frames, const Ellipse& e, int bw, int bh,
                        const PhaseRef& ref, float* out, float* stds_out, cudaStream_t st);

// Host side (shape.cu).
// Block-map Hu metric: the bw x bh reference patch (ellipse pixels of the
// ReferenceBlock2D normalised like the kernel's comparison patches) and its
// Hu invariant 1.
void hu_prepare_patch(const float* ref_pixels, int bw, int bh, float* grid);
double patch_hu1(const float* patch, int bw, int bh);
// Block-map phase metric: DFT of the reference block.
void phase_reference_dft(const float* ref_pixels, float ref_std, int bw, int bh, PhaseRef* out);

}  // namespace sred
