/*
 * CPU oracle for the SReD block-correlation path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (libsred, the Python
 * package) links, loads or calls this file; only tests/, the smoke check and
 * the CPU-baseline leg of bench.py do, and only as the checker.
 *
 * Two restatements of the reference's arithmetic live here:
 *
 *  - "f32": the reference's FP32 semantics, statement for statement in the
 *    same evaluation order, so that on an IEEE-754 host without FMA
 *    contraction it reproduces the reference kernels and the Java host code
 *    bit for bit (checked against the reference's own kernels compiled by
 *    oracle/refshim, and against the reference's JUnit golden vectors).
 *    The order of operations is kept identical on purpose: bit parity with
 *    FP32 code depends on it.
 *
 *  - "f64": an independent double-precision evaluation of the same maps.
 *    Discrete decisions (relevance: sigma^2 < threshold; flatness:
 *    sigma == 0) are taken on the reference's FP32 local statistics, which
 *    the caller passes in, so the f64 result is "the reference's maps
 *    computed exactly"; every continuous quantity (block moments, weights,
 *    covariances, the per-pixel division) is FP64.
 *
 * Reference files cited below are relative to the SReD repository root:
 *   cl/   = src/main/resources/
 *   java/ = src/main/java/
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EPS 0.0000001f /* java/Utils.java:20 (Utils.EPSILON) */

enum { ORC_PEARSON = 0, ORC_SSIM = 1, ORC_NRMSE = 2, ORC_ABSDIFF = 3, ORC_COSINE = 4 };

/* ------------------------------------------------------------------ */
/* Java float semantics helpers                                        */
/* ------------------------------------------------------------------ */

/* java.lang.Math.min(float,float): NaN-propagating, -0.0f < +0.0f. */
static float jmin(float a, float b) {
    if (a != a) return a;
    if (a == 0.0f && b == 0.0f) return signbit(a) ? a : b;
    return a <= b ? a : b;
}
/* java.lang.Math.max(float,float). */
static float jmax(float a, float b) {
    if (a != a) return a;
    if (a == 0.0f && b == 0.0f) return signbit(a) ? b : a;
    return a >= b ? a : b;
}

/* Inscribed-ellipse membership test used for every block gather
 * (java/GlobalRepetition2D_.java:102-111, cl/kernelGetLocalStatistics2D.cl:31-33). */
static int in_ellipse(int dx, int dy, int rw, int rh) {
    float fx = (float)dx, fy = (float)dy;
    return ((fx * fx) / (float)(rw * rw)) + ((fy * fy) / (float)(rh * rh)) <= 1.0f;
}

int orc_block_size(int bw, int bh) {
    int rw = bw / 2, rh = bh / 2, k = 0;
    for (int y = 0; y < bh; y++)
        for (int x = 0; x < bw; x++)
            if (in_ellipse(x - rw, y - rh, rw, rh)) k++;
    return k;
}

/* Pixel offsets (row-major ellipse order) of a block, relative to its centre. */
static int ellipse_offsets(int bw, int bh, int W, int *off) {
    int rw = bw / 2, rh = bh / 2, k = 0;
    for (int y = -rh; y <= rh; y++)
        for (int x = -rw; x <= rw; x++)
            if (in_ellipse(x, y, rw, rh)) off[k++] = y * W + x;
    return k;
}

/* ------------------------------------------------------------------ */
/* a3: local statistics, cl/kernelGetLocalStatistics2D.cl:15-56         */
/* ------------------------------------------------------------------ */
void orc_local_stats_f32(const float *img, int W, int H, int bw, int bh,
                         float *means, float *stds) {
    int rw = bw / 2, rh = bh / 2;
    int *off = (int *)malloc(sizeof(int) * bw * bh);
    int K = ellipse_offsets(bw, bh, W, off);
    #pragma omp parallel for schedule(static)
    for (int gy = 0; gy < H; gy++) {
        float blk[1024];
        for (int gx = 0; gx < W; gx++) {
            int p = gy * W + gx;
            if (gx < rw || gx >= W - rw || gy < rh || gy >= H - rh) {
                means[p] = 0.0f; stds[p] = 0.0f; continue;
            }
            for (int i = 0; i < K; i++) blk[i] = img[p + off[i]];
            float mean = 0.0f;
            for (int i = 0; i < K; i++) mean += blk[i];
            mean /= (float)K;
            means[p] = mean;
            float var = 0.0f;
            for (int i = 0; i < K; i++) var += (blk[i] - mean) * (blk[i] - mean);
            var /= (float)(K - 1);
            stds[p] = sqrtf(var);
        }
    }
    free(off);
}

/* ------------------------------------------------------------------ */
/* a1: min-max normalisation of the input image, java/Utils.java:707-722 */
/* ------------------------------------------------------------------ */
void orc_normalize_input(float *img, int n) {
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int i = 0; i < n; i++) { mn = jmin(mn, img[i]); mx = jmax(mx, img[i]); }
    for (int i = 0; i < n; i++) img[i] = (img[i] - mn) / (mx - mn + ORC_EPS);
}

/* ------------------------------------------------------------------ */
/* a4: noise variance, java/Utils.java:790-837 and :854-900             */
/* Returns 0 on success, -1 where the reference throws (no tile).       */
/* ------------------------------------------------------------------ */
static int cmp_float(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

int orc_mean_noise_var(const float *img, int W, int H, float *out) {
    int wh = W * H, t = (wh <= 352 * 288) ? 8 : 16;
    int nbx = W / t, nby = H / t, nb = nbx * nby;
    float *vars = (float *)malloc(sizeof(float) * (nb > 0 ? nb : 1));
    int idx = 0;
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            float mean = 0.0f, sq = 0.0f;
            for (int y = by * t; y < (by + 1) * t; y++)
                for (int x = bx * t; x < (bx + 1) * t; x++) {
                    float v = img[y * W + x];
                    mean += v;
                    sq += v * v;
                }
            mean /= (float)(t * t);
            vars[idx++] = sq / (float)(t * t) - mean * mean;
        }
    qsort(vars, nb, sizeof(float), cmp_float);
    int nv = (int)(0.03f * (float)nb + 1.0f);
    if (nv > nb) { free(vars); return -1; } /* ArrayIndexOutOfBounds in the reference */
    float nvar = 0.0f;
    for (int i = 0; i < nv; i++) nvar += vars[i];
    nvar = fabsf(nvar / (float)nv);
    nvar = (1.0f + 0.001f * (nvar - 40.0f)) * nvar;
    free(vars);
    *out = nvar;
    return 0;
}

/* a5: relevance mask, java/Utils.java:944-968. Returns -1 like a4. */
int orc_relevance_mask(const float *img, int W, int H, int rw, int rh, const float *stds,
                       float c, float *mask, float *threshold, float *noise_var) {
    float v;
    if (orc_mean_noise_var(img, W, H, &v) != 0) return -1;
    float thr = v * c;
    memset(mask, 0, sizeof(float) * (size_t)W * H);
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            float s = stds[y * W + x];
            mask[y * W + x] = (s * s) <= thr ? 0.0f : 1.0f;
        }
    *threshold = thr;
    *noise_var = v;
    return 0;
}

/* java/Utils.java:985-1031. mask may be NULL. Returns -1 for a non-binary mask. */
int orc_normalize_image(float *a, int W, int H, int bw_, int bh_, const float *mask) {
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int y = bh_; y < H - bh_; y++)
        for (int x = bw_; x < W - bw_; x++) {
            int i = y * W + x;
            if (mask) {
                if (mask[i] != 0.0f && mask[i] != 1.0f) return -1;
                if (!(mask[i] > 0.0f)) continue;
            }
            mn = jmin(a[i], mn);
            mx = jmax(a[i], mx);
        }
    for (int y = bh_; y < H - bh_; y++)
        for (int x = bw_; x < W - bw_; x++) {
            int i = y * W + x;
            if (mask && !(mask[i] > 0.0f)) continue;
            a[i] = (a[i] - mn) / (mx - mn + ORC_EPS);
        }
    return 0;
}

/* java/Utils.java:919-930 */
void orc_apply_mask(float *a, int n, const float *mask) {
    for (int i = 0; i < n; i++) a[i] *= mask[i];
}

/* a6: java/GlobalRepetition2D_.java:133-140 */
float orc_n_pixels(const float *mask, int W, int H, int rw, int rh) {
    float n = 0.0f;
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++)
            if (mask[y * W + x] > 0.0f) n += 1.0f;
    return n;
}

/* ------------------------------------------------------------------ */
/* a7-a10: global kernels, FP32 reference semantics.                   */
/* cl/kernelGetGlobalPearson2D.cl:11-110, cl/kernelGetGlobalSsim2D.cl, */
/* cl/kernelGetGlobalNrmse2D.cl, cl/kernelGetGlobalAbsDiffStds2D.cl.   */
/* Evaluates the reference pixels listed in `pix` (n_pix of them);    */
/* num/den are indexed like pix. A reference pixel on the border or    */
/* below threshold gets num = den = 0, as the reference leaves it.     */
/* ------------------------------------------------------------------ */
void orc_global_f32(int metric, const float *img, int W, int H, int bw, int bh,
                    const float *means, const float *stds, float filter_param, float threshold,
                    const int *pix, int n_pix, float *num, float *den) {
    int rw = bw / 2, rh = bh / 2;
    int *off = (int *)malloc(sizeof(int) * bw * bh);
    int K = ellipse_offsets(bw, bh, W, off);
    const float c1 = 0.0001f, c2 = 0.0009f;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int ii = 0; ii < n_pix; ii++) {
        int p = pix[ii], gx = p % W, gy = p / W;
        float S = 0.0f, Wsum = 0.0f;
        float rb[1024], tb[1024];
        if (gx < rw || gx >= W - rw || gy < rh || gy >= H - rh) { num[ii] = 0; den[ii] = 0; continue; }
        float rs = stds[p];
        if (rs * rs < threshold) { num[ii] = 0; den[ii] = 0; continue; }
        float rm = means[p];
        if (metric != ORC_ABSDIFF)
            for (int i = 0; i < K; i++) rb[i] = img[p + off[i]] - rm;
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                int q = y * W + x;
                float ts = stds[q];
                if (ts * ts < threshold) continue;
                float wgt = expf((-1.0f) * (((rs - ts) * (rs - ts)) / (filter_param + ORC_EPS)));
                if (metric == ORC_ABSDIFF) {
                    Wsum += wgt;
                    S += fabsf(rs - ts) * wgt;
                    continue;
                }
                float tm = means[q];
                for (int i = 0; i < K; i++) tb[i] = img[q + off[i]] - tm;
                if (metric == ORC_NRMSE) {
                    Wsum += wgt;
                    float mse = 0.0f;
                    for (int i = 0; i < K; i++) mse += (rb[i] - tb[i]) * (rb[i] - tb[i]);
                    mse /= (float)K;
                    S += sqrtf(mse);
                    continue;
                }
                float cov = 0.0f;
                for (int i = 0; i < K; i++) cov += rb[i] * tb[i];
                cov /= (float)(K - 1);
                Wsum += wgt;
                if (rs == 0.0f && ts == 0.0f) {
                    S += 1.0f * wgt;
                } else if (rs == 0.0f || ts == 0.0f) {
                    S += 0.0f;
                } else if (metric == ORC_PEARSON) {
                    S += fmaxf(0.0f, cov / ((rs * ts) + ORC_EPS)) * wgt;
                } else { /* SSIM, with the product (mu_p^2 * mu_q^2) in the denominator */
                    float ssim = ((2.0f * rm * tm + c1) * (2.0f * cov + c2)) /
                                 (((rm * rm) * (tm * tm) + c1) * ((rs * rs) + (ts * ts) + c2)) * wgt;
                    S += fmaxf(0.0f, ssim);
                }
            }
        num[ii] = S;
        den[ii] = Wsum;
    }
    free(off);
}

/* ------------------------------------------------------------------ */
/* Global kernels, FP64 evaluation (the judge).                        */
/* Decisions use the FP32 stds passed in; values are FP64.             */
/* ------------------------------------------------------------------ */
void orc_global_f64(int metric, const float *img, int W, int H, int bw, int bh,
                    const float *stds32, float filter_param, float threshold,
                    const int *pix, int n_pix, double *num, double *den) {
    int rw = bw / 2, rh = bh / 2;
    int *off = (int *)malloc(sizeof(int) * bw * bh);
    int K = ellipse_offsets(bw, bh, W, off);
    int nx = W - 2 * rw, ny = H - 2 * rh;
    /* Relevant test blocks: FP64 moments and centred vectors, computed once. */
    int nq = 0;
    int *qi = (int *)malloc(sizeof(int) * (size_t)(nx > 0 && ny > 0 ? nx * ny : 1));
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            float s = stds32[y * W + x];
            if (!(s * s < threshold)) qi[nq++] = y * W + x;
        }
    double *qv = (double *)malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1) * K);
    double *qm = (double *)malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1));
    double *qs = (double *)malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1));
    #pragma omp parallel for schedule(static)
    for (int j = 0; j < nq; j++) {
        int q = qi[j];
        double m = 0.0, v = 0.0;
        for (int i = 0; i < K; i++) m += (double)img[q + off[i]];
        m /= K;
        for (int i = 0; i < K; i++) {
            double d = (double)img[q + off[i]] - m;
            qv[(size_t)j * K + i] = d;
            v += d * d;
        }
        qm[j] = m;
        qs[j] = sqrt(v / (K - 1));
    }
    const double c1 = (double)0.0001f, c2 = (double)0.0009f;
    const double h = (double)filter_param + (double)ORC_EPS;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int ii = 0; ii < n_pix; ii++) {
        int p = pix[ii], gx = p % W, gy = p / W;
        num[ii] = 0; den[ii] = 0;
        if (gx < rw || gx >= W - rw || gy < rh || gy >= H - rh) continue;
        float rs32 = stds32[p];
        if (rs32 * rs32 < threshold) continue;
        double rb[1024], rm = 0.0, rv = 0.0;
        for (int i = 0; i < K; i++) rm += (double)img[p + off[i]];
        rm /= K;
        for (int i = 0; i < K; i++) { rb[i] = (double)img[p + off[i]] - rm; rv += rb[i] * rb[i]; }
        double rs = sqrt(rv / (K - 1));
        double S = 0.0, Ws = 0.0;
        for (int j = 0; j < nq; j++) {
            const double *tb = qv + (size_t)j * K;
            double ts = qs[j], tm = qm[j];
            double wgt = exp(-((rs - ts) * (rs - ts)) / h);
            Ws += wgt;
            if (metric == ORC_ABSDIFF) { S += fabs(rs - ts) * wgt; continue; }
            if (metric == ORC_NRMSE) {
                double mse = 0.0;
                for (int i = 0; i < K; i++) { double d = rb[i] - tb[i]; mse += d * d; }
                S += sqrt(mse / K);
                continue;
            }
            int f_r = (rs32 == 0.0f), f_t = (stds32[qi[j]] == 0.0f);
            if (f_r && f_t) { S += wgt; continue; }
            if (f_r || f_t) continue;
            double cov = 0.0;
            for (int i = 0; i < K; i++) cov += rb[i] * tb[i];
            cov /= (K - 1);
            if (metric == ORC_PEARSON) {
                double r = cov / (rs * ts + (double)ORC_EPS);
                S += (r > 0.0 ? r : 0.0) * wgt;
            } else {
                double s = ((2.0 * rm * tm + c1) * (2.0 * cov + c2)) /
                           ((rm * rm * tm * tm + c1) * (rs * rs + ts * ts + c2)) * wgt;
                S += s > 0.0 ? s : 0.0;
            }
        }
        num[ii] = S;
        den[ii] = Ws;
    }
    free(off); free(qi); free(qv); free(qm); free(qs);
}

/* ------------------------------------------------------------------ */
/* a11: host finalisation, java/CLUtils.java:1747-1770 (Pearson/SSIM), */
/* :1998-2027 (NRMSE), :2127-2156 (Abs-diff). Operates in place on a   */
/* full W*H map whose interior holds num, with den alongside.          */
/* ------------------------------------------------------------------ */
int orc_global_finalize_f32(int metric, const float *num, const float *den, int W, int H,
                            int rw, int rh, const float *mask, float relevance_constant,
                            float n_pixels, int normalize, float *out) {
    memset(out, 0, sizeof(float) * (size_t)W * H);
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            int i = y * W + x;
            out[i] = num[i] / (den[i] * n_pixels + ORC_EPS);
        }
    if (metric == ORC_NRMSE || metric == ORC_ABSDIFF) {
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                int i = y * W + x;
                if (mask[i] > 0.0f) out[i] = (out[i] == 0.0f) ? 1.0f : 1.0f / out[i];
            }
    }
    if (relevance_constant > 0.0f) orc_apply_mask(out, W * H, mask);
    if (normalize) return orc_normalize_image(out, W, H, rw, rh, mask);
    return 0;
}

/* FP64 finalisation of the FP64 sums (the judge's normalised map). */
void orc_global_finalize_f64(int metric, const double *num, const double *den, int W, int H,
                             int rw, int rh, const float *mask, float relevance_constant,
                             double n_pixels, int normalize, double *out) {
    memset(out, 0, sizeof(double) * (size_t)W * H);
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            int i = y * W + x;
            out[i] = num[i] / (den[i] * n_pixels + (double)ORC_EPS);
            if ((metric == ORC_NRMSE || metric == ORC_ABSDIFF) && mask[i] > 0.0f)
                out[i] = (out[i] == 0.0) ? 1.0 : 1.0 / out[i];
        }
    if (relevance_constant > 0.0f)
        for (int i = 0; i < W * H; i++) out[i] *= (double)mask[i];
    if (!normalize) return;
    double mn = DBL_MAX, mx = -DBL_MAX;
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            int i = y * W + x;
            if (!(mask[i] > 0.0f)) continue;
            if (out[i] < mn) mn = out[i];
            if (out[i] > mx) mx = out[i];
        }
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            int i = y * W + x;
            if (mask[i] > 0.0f) out[i] = (out[i] - mn) / (mx - mn + (double)ORC_EPS);
        }
}

/* ------------------------------------------------------------------ */
/* a13: reference block from a block image, java/Utils.java:557-639.   */
/* Returns K; pixels receives K values; mean/std as the reference      */
/* stores them (the std subtracts the mean a second time).             */
/* ------------------------------------------------------------------ */
int orc_reference_block(const float *blk, int bw, int bh, float *pixels, float *mean_out,
                        float *std_out) {
    int rw = bw / 2, rh = bh / 2, K = 0;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            if (in_ellipse(i - rw, j - rh, rw, rh)) pixels[K++] = blk[j * bw + i];
    float mn = FLT_MAX, mx = -FLT_MAX;
    for (int i = 0; i < K; i++) { mn = jmin(mn, pixels[i]); mx = jmax(mx, pixels[i]); }
    float mean = 0.0f;
    for (int i = 0; i < K; i++) {
        pixels[i] = (pixels[i] - mn) / (mx - mn + ORC_EPS);
        mean += pixels[i];
    }
    mean /= (float)K;
    for (int i = 0; i < K; i++) pixels[i] = pixels[i] - mean;
    float sd = 0.0f;
    for (int i = 0; i < K; i++) sd += (pixels[i] - mean) * (pixels[i] - mean);
    sd = (float)sqrt((double)(sd / ((float)(K - 1))));
    *mean_out = mean;
    *std_out = sd;
    return K;
}

/* ------------------------------------------------------------------ */
/* a14: block (local) repetition map kernels, FP32 reference semantics. */
/* cl/kernelGetBlockPearson2D.cl:34-89, cl/kernelGetBlockSsim2D.cl:74-80,*/
/* cl/kernelGetBlockNrmse2D.cl:69-74, cl/kernelGetBlockAbsDiffStds2D.cl.*/
/* ------------------------------------------------------------------ */
void orc_block_kernel_f32(int metric, const float *img, int W, int H, int bw, int bh,
                          const float *means, const float *stds, const float *ref, int K,
                          float ref_mean, float ref_std, float *map) {
    int rw = bw / 2, rh = bh / 2;
    int *off = (int *)malloc(sizeof(int) * bw * bh);
    ellipse_offsets(bw, bh, W, off);
    const float c1 = 0.0001f, c2 = 0.0009f;
    #pragma omp parallel for schedule(static)
    for (int gy = 0; gy < H; gy++) {
        float cb[1024];
        for (int gx = 0; gx < W; gx++) {
            int p = gy * W + gx;
            if (gx < rw || gx >= W - rw || gy < rh || gy >= H - rh) { map[p] = 0.0f; continue; }
            float ts = stds[p];
            if (metric == ORC_ABSDIFF) { map[p] = fabsf(ref_std - ts); continue; }
            float cm = means[p];
            for (int i = 0; i < K; i++) cb[i] = img[p + off[i]] - cm;
            if (metric == ORC_NRMSE) {
                float mse = 0.0f;
                for (int i = 0; i < K; i++) mse += (ref[i] - cb[i]) * (ref[i] - cb[i]);
                mse /= (float)K;
                map[p] = sqrtf(mse);
                continue;
            }
            float cov = 0.0f;
            for (int i = 0; i < K; i++) cov += ref[i] * cb[i];
            cov /= (float)(K - 1);
            if (ref_std == 0.0f && ts == 0.0f) map[p] = 1.0f;
            else if (ref_std == 0.0f || ts == 0.0f) map[p] = 0.0f;
            else if (metric == ORC_PEARSON) map[p] = fmaxf(0.0f, cov / ((ref_std * ts) + ORC_EPS));
            else {
                float s = ((2.0f * ref_mean * cm + c1) * (2.0f * cov + c2)) /
                          (((ref_mean * ref_mean) + (cm * cm) + c1) * ((ref_std * ref_std) + (ts * ts) + c2));
                map[p] = fmaxf(0.0f, s);
            }
        }
    }
    free(off);
}

/* Block-map host post-processing, java/CLUtils.java:564-577 (Pearson, SSIM),
 * :788-841 (NRMSE), :928-975 (Abs-diff). `map` holds the kernel output and is
 * finished in place. Returns -1 where the reference throws. */
int orc_block_postprocess_f32(int metric, float *map, const float *img, int W, int H, int rw,
                              int rh, const float *stds, float c, int normalize) {
    size_t n = (size_t)W * H;
    float *mask = NULL;
    float thr, nv;
    int rc = 0;
    if (metric == ORC_NRMSE) {
        mask = (float *)calloc(n, sizeof(float));
        if (c == 0.0f) {
            for (int y = rh; y < H - rh; y++)
                for (int x = rw; x < W - rw; x++) mask[y * W + x] = 1.0f;
        } else if (orc_relevance_mask(img, W, H, rw, rh, stds, c, mask, &thr, &nv) != 0) {
            free(mask);
            return -1;
        }
        orc_apply_mask(map, (int)n, mask);
        orc_normalize_image(map, W, H, rw, rh, mask);
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                int i = y * W + x;
                if (mask[i] > 0.0f) map[i] = (map[i] == 0.0f) ? 1.0f : 1.0f / map[i];
            }
        if (normalize) rc = orc_normalize_image(map, W, H, rw, rh, mask);
        free(mask);
        return rc;
    }
    if (metric == ORC_ABSDIFF) {
        float mn = FLT_MAX, mx = 1.4e-45f; /* Float.MIN_VALUE, java/CLUtils.java:940 */
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                mn = jmin(mn, map[y * W + x]);
                mx = jmax(mx, map[y * W + x]);
            }
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                int i = y * W + x;
                map[i] = (map[i] - mn) / (mx - mn + ORC_EPS);
            }
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) map[y * W + x] = 1.0f - map[y * W + x];
    }
    if (c > 0.0f) {
        mask = (float *)calloc(n, sizeof(float));
        if (orc_relevance_mask(img, W, H, rw, rh, stds, c, mask, &thr, &nv) != 0) {
            free(mask);
            return -1;
        }
        orc_apply_mask(map, (int)n, mask);
    }
    if (normalize) rc = orc_normalize_image(map, W, H, rw, rh, mask);
    free(mask);
    return rc;
}

/* FP64 block-map kernel: the judge for the block maps, including the metrics
 * the reference does not ship in working form.
 *   cosine  = <x_p, r> / (|x_p| |r| + eps) on raw (not centred) ellipse vectors;
 *   Pearson/SSIM/NRMSE/Abs-diff as the reference kernels, with FP64 moments of
 *   the comparison block and the flat-block decisions taken on the FP32 stds. */
void orc_block_kernel_f64(int metric, const float *img, int W, int H, int bw, int bh,
                          const float *stds32, const float *ref, int K, float ref_mean,
                          float ref_std, double *map) {
    int rw = bw / 2, rh = bh / 2;
    int *off = (int *)malloc(sizeof(int) * bw * bh);
    ellipse_offsets(bw, bh, W, off);
    const double c1 = (double)0.0001f, c2 = (double)0.0009f;
    #pragma omp parallel for schedule(static)
    for (int gy = 0; gy < H; gy++) {
        double cb[1024];
        for (int gx = 0; gx < W; gx++) {
            int p = gy * W + gx;
            map[p] = 0.0;
            if (gx < rw || gx >= W - rw || gy < rh || gy >= H - rh) continue;
            double cm = 0.0, cv = 0.0;
            for (int i = 0; i < K; i++) cm += (double)img[p + off[i]];
            cm /= K;
            for (int i = 0; i < K; i++) { cb[i] = (double)img[p + off[i]] - cm; cv += cb[i] * cb[i]; }
            double ts = sqrt(cv / (K - 1));
            if (metric == ORC_ABSDIFF) { map[p] = fabs((double)ref_std - ts); continue; }
            if (metric == ORC_COSINE) {
                double d = 0.0, nr = 0.0, nc = 0.0;
                for (int i = 0; i < K; i++) {
                    double a = (double)ref[i], b = (double)img[p + off[i]];
                    d += a * b; nr += a * a; nc += b * b;
                }
                map[p] = d / (sqrt(nr) * sqrt(nc) + (double)ORC_EPS);
                continue;
            }
            if (metric == ORC_NRMSE) {
                double mse = 0.0;
                for (int i = 0; i < K; i++) { double d = (double)ref[i] - cb[i]; mse += d * d; }
                map[p] = sqrt(mse / K);
                continue;
            }
            double cov = 0.0;
            for (int i = 0; i < K; i++) cov += (double)ref[i] * cb[i];
            cov /= (K - 1);
            float ts32 = stds32[p];
            if (ref_std == 0.0f && ts32 == 0.0f) { map[p] = 1.0; continue; }
            if (ref_std == 0.0f || ts32 == 0.0f) continue;
            double r;
            if (metric == ORC_PEARSON) {
                r = cov / ((double)ref_std * ts + (double)ORC_EPS);
            } else {
                double rm = (double)ref_mean, rs = (double)ref_std;
                r = ((2.0 * rm * cm + c1) * (2.0 * cov + c2)) /
                    ((rm * rm + cm * cm + c1) * (rs * rs + ts * ts + c2));
            }
            map[p] = r > 0.0 ? r : 0.0;
        }
    }
    free(off);
}

/* java.util.Random: the published 48-bit LCG (seed scrambling with
 * 0x5DEECE66D, next(bits), nextFloat() = next(24) / 2^24). Used to rebuild
 * the reference's seeded test inputs. */
void orc_java_random_floats(int64_t seed, int n, float *out) {
    uint64_t s = ((uint64_t)seed ^ 0x5DEECE66DULL) & ((1ULL << 48) - 1);
    for (int i = 0; i < n; i++) {
        s = (s * 0x5DEECE66DULL + 0xBULL) & ((1ULL << 48) - 1);
        int32_t bits = (int32_t)(s >> (48 - 24));
        out[i] = (float)bits / (float)(1 << 24);
    }
}
