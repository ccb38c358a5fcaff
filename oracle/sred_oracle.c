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

/* ------------------------------------------------------------------ */
/* Shape metrics: Hu moments and phase correlation                     */
/*                                                                     */
/* The reference ships three OpenCL kernels for these that its Java    */
/* code never loads: cl/kernelGetPatchHu2D.cl (one patch against every */
/* block, FP64), cl/kernelGetHuMap.cl (all pairs, FP32) and            */
/* cl/kernelGetPhaseCorrelationMap.cl (all pairs, FP64; it does not    */
/* compile as shipped). The functions below restate them statement for */
/* statement. $PATCH_SIZE$ is the ellipse count K for the Hu patch     */
/* kernel (the Java convention, java/RelevanceMask2D_.java:161-167)    */
/* and bw*bh for the two all-pairs kernels, whose private arrays hold  */
/* the whole square block. The phase kernel is restated with three     */
/* repairs: no unique-coordinate pre-filter (its nUnique is never      */
/* defined, :27), real-valued DFT phases (the shipped (1*i*ii/bW) is   */
/* an integer division, :66/:101/:138) and the peak search indexed     */
/* with the block width (the shipped j*w+i reads past the block,       */
/* :150).                                                              */
/* ------------------------------------------------------------------ */

/* cl/kernelGetPatchHu2D.cl:38-40 (float test) and :58-60 (double test);
 * both select the same positions as in_ellipse() for every odd size 3..15. */
static int hu_in_ellipse_f(int i, int j, int rw, int rh) {
    float dx = (float)(i - rw) / rw, dy = (float)(j - rh) / rh;
    return dx * dx + dy * dy <= 1.0f;
}

/* Hu invariant 1 of a bw x bh patch read at the ellipse positions:
 * cl/kernelGetPatchHu2D.cl:51-101 (reference patch) = :189-239 (comparison
 * patch). Raw moments use 1-based coordinates, central moments 0-based
 * ones, as the kernel does. */
static double orc_hu1_patch(const double *v, int bw, int bh) {
    const int rw = bw / 2, rh = bh / 2;
    double M00 = 0.0, M10 = 0.0, M01 = 0.0;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            if (hu_in_ellipse_f(i, j, rw, rh)) {
                double p = v[j * bw + i];
                M00 += p;
                M10 += (double)(i + 1) * p;
                M01 += (double)(j + 1) * p;
            }
    double cx = M10 / (M00 + (double)ORC_EPS);
    double cy = M01 / (M00 + (double)ORC_EPS);
    double mu20 = 0.0, mu02 = 0.0;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            if (hu_in_ellipse_f(i, j, rw, rh)) {
                double p = v[j * bw + i];
                mu20 += pow(((double)i - cx), 2.0) * p;
                mu02 += pow(((double)j - cy), 2.0) * p;
            }
    double nu20 = mu20 / (pow(M00, 2.0) + (double)ORC_EPS);
    double nu02 = mu02 / (pow(M00, 2.0) + (double)ORC_EPS);
    return nu20 + nu02;
}

/* Hu invariant 1 of the reference patch as the kernel reads it
 * (cl/kernelGetPatchHu2D.cl:34-44: float patch values widened to double). */
double orc_patch_hu1_ref(const float *patch, int bw, int bh) {
    double v[32 * 32];
    if (bw > 31 || bh > 31) return NAN;
    for (int k = 0; k < bw * bh; k++) v[k] = (double)patch[k];
    return orc_hu1_patch(v, bw, bh);
}

/* cl/kernelGetPatchHu2D.cl:18-267 for every pixel: interior pixels get
 * (float)sqrt(hu1_ref * hu1_comp), border pixels are left untouched. */
void orc_patch_hu(const float *patch, const float *img, int W, int H, int bw, int bh, int patch_size,
                  float *out) {
    const int rw = bw / 2, rh = bh / 2;
    const double ref_hu1 = orc_patch_hu1_ref(patch, bw, bh);
    double comp[32 * 32];
    for (int gy = rh; gy < H - rh; gy++)
        for (int gx = rw; gx < W - rw; gx++) {
            double mean = 0.0;
            /* :129-140, the gather's ellipse test divides integers, so it keeps
             * every position of the square except its four corners */
            for (int j = gy - rh; j <= gy + rh; j++)
                for (int i = gx - rw; i <= gx + rw; i++) {
                    float dx = (float)((i - gx) / rw);
                    float dy = (float)((j - gy) / rh);
                    if (dx * dx + dy * dy <= 1.0f) {
                        double p = (double)img[j * W + i];
                        comp[(j - (gy - rh)) * bw + (i - (gx - rw))] = p;
                        mean += p;
                    }
                }
            mean /= (double)patch_size;
            for (int j = 0; j < bh; j++) /* :143-151 */
                for (int i = 0; i < bw; i++)
                    if (hu_in_ellipse_f(i, j, rw, rh)) comp[j * bw + i] -= mean;
            double mn = DBL_MAX, mx = -DBL_MAX; /* :158-171 */
            for (int j = 0; j < bh; j++)
                for (int i = 0; i < bw; i++)
                    if (hu_in_ellipse_f(i, j, rw, rh)) {
                        double p = comp[j * bw + i];
                        mn = p < mn ? p : mn;
                        mx = p > mx ? p : mx;
                    }
            for (int j = 0; j < bh; j++) /* :174-182 */
                for (int i = 0; i < bw; i++)
                    if (hu_in_ellipse_f(i, j, rw, rh))
                        comp[j * bw + i] = (comp[j * bw + i] - mn) / (mx - mn + (double)ORC_EPS);
            out[gy * W + gx] = (float)sqrt(ref_hu1 * orc_hu1_patch(comp, bw, bh));
        }
}

/* Reference patch of the block-map form of the Hu metric (a definition of
 * this library; the reference never wires the kernel): the ReferenceBlock2D
 * pixels (ellipse order) scattered onto the bw x bh grid and normalised the
 * way cl/kernelGetPatchHu2D.cl:126-182 normalises every comparison patch
 * (mean-subtract over the ellipse, then min-max to [0, 1]), in FP64, stored
 * as float like the kernel's patch buffer. Off-ellipse grid cells are 0. */
void orc_hu_prepare_patch(const float *ref_pixels, int bw, int bh, float *grid) {
    const int rw = bw / 2, rh = bh / 2;
    double v[32 * 32];
    int k = 0, K = 0;
    double mean = 0.0;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            if (hu_in_ellipse_f(i, j, rw, rh)) K++;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++) {
            v[j * bw + i] = 0.0;
            if (hu_in_ellipse_f(i, j, rw, rh)) {
                v[j * bw + i] = (double)ref_pixels[k++];
                mean += v[j * bw + i];
            }
        }
    mean /= (double)K;
    double mn = DBL_MAX, mx = -DBL_MAX;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            if (hu_in_ellipse_f(i, j, rw, rh)) {
                v[j * bw + i] -= mean;
                mn = v[j * bw + i] < mn ? v[j * bw + i] : mn;
                mx = v[j * bw + i] > mx ? v[j * bw + i] : mx;
            }
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            grid[j * bw + i] = hu_in_ellipse_f(i, j, rw, rh)
                                   ? (float)((v[j * bw + i] - mn) / (mx - mn + (double)ORC_EPS))
                                   : 0.0f;
}

/* getInvariant (cl/kernelGetHuMap.cl:146-172), FP32. */
static float orc_hu_invariant(const float *patch, int pw, int ph, int p, int q) {
    float x_avg = 0.0f;
    for (int i = 1; i <= pw; i++) x_avg += (float)i;
    x_avg /= (float)pw;
    float y_avg = 0.0f;
    for (int i = 1; i <= ph; i++) y_avg += (float)i;
    y_avg /= (float)ph;
    float mu_pq = 0.0f, mu_00 = 0.0f;
    for (int j = 0; j < ph; j++)
        for (int i = 0; i < pw; i++) {
            mu_pq += (float)powf((float)i + 1.0f - x_avg, (float)p) *
                     ((float)powf((float)j + 1.0f - y_avg, (float)q)) * patch[j * pw + i];
            mu_00 += patch[j * pw + i];
        }
    mu_00 = (float)powf(mu_00, 1.0f + (p + q) / 2.0f);
    return mu_pq / (mu_00 + ORC_EPS);
}

/* Per-block Hu feature of cl/kernelGetHuMap.cl:62-80 (= :109-124): the whole
 * square block minus the block's local mean, invariant(2,0) + invariant(0,2). */
float orc_hu_feature(const float *img, const float *means, int W, int bw, int bh, int x0, int y0) {
    float patch[32 * 32];
    const int rw = bw / 2, rh = bh / 2;
    const float m = means[y0 * W + x0];
    int c = 0;
    for (int j = y0 - rh; j <= y0 + rh; j++)
        for (int i = x0 - rw; i <= x0 + rw; i++) patch[c++] = img[j * W + i] - m;
    return orc_hu_invariant(patch, bw, bh, 2, 0) + orc_hu_invariant(patch, bw, bh, 0, 2);
}

/* getExpDecayWeight of cl/kernelGetHuMap.cl:136-144. */
static float orc_hu_weight(float ref, float comp) {
    float similarity = 1.0f - (fabsf(ref - comp) / (fabsf(ref) + fabsf(comp) + ORC_EPS));
    return ((float)powf(100.0f, similarity) - 1) / 99;
}

/* cl/kernelGetHuMap.cl:23-133 for every interior reference pixel:
 * sum over every interior q of |hu_q - hu_p| * weight(sigma_p, sigma_q).
 * f64acc = 0: the reference's FP32 accumulation in raster order;
 * f64acc = 1: the same FP32 terms summed in FP64 (the judge). */
void orc_hu_map(const float *img, const float *means, const float *stds, int W, int H, int bw, int bh,
                int f64acc, double *out) {
    const int rw = bw / 2, rh = bh / 2;
    float *feat = (float *)calloc((size_t)W * H, sizeof(float));
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) feat[y * W + x] = orc_hu_feature(img, means, W, bw, bh, x, y);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int y0 = rh; y0 < H - rh; y0++)
        for (int x0 = rw; x0 < W - rw; x0++) {
            const float ref_hu = feat[y0 * W + x0];
            float acc32 = 0.0f;
            double acc64 = 0.0;
            for (int y1 = rh; y1 < H - rh; y1++)
                for (int x1 = rw; x1 < W - rw; x1++) {
                    float weight = orc_hu_weight(stds[y0 * W + x0], stds[y1 * W + x1]);
                    float t = fabsf((float)feat[y1 * W + x1] - (float)ref_hu) * weight;
                    acc32 += t;
                    acc64 += (double)t;
                }
            out[y0 * W + x0] = f64acc ? acc64 : (double)acc32;
        }
    free(feat);
}

/* The kernel's pi is a float literal widened to double
 * (cl/kernelGetPhaseCorrelationMap.cl:44). */
static const double ORC_PHASE_PI = (double)3.14159265358979323846f;

/* Forward DFT of a bw x bh real patch, as :59-71 / :93-106 compute it (with
 * real-valued phases). tc/ts: cos/sin tables of the n x n phase matrix. */
static void orc_phase_dft(const double *x, int n, const double *tc, const double *ts, double *re, double *im) {
    const double sn = sqrt((double)n);
    for (int a = 0; a < n; a++) {
        re[a] = 0.0;
        im[a] = 0.0;
        for (int b = 0; b < n; b++) {
            re[a] += (x[b] * tc[a * n + b]) / sn;
            im[a] -= (x[b] * ts[a * n + b]) / sn;
        }
    }
}

/* Phase tables: angle(a = j*bw+i, b = jj*bw+ii) = 2*PI*((1.0*i*ii/bw) + (1.0*j*jj/bh)). */
static void orc_phase_tables(int bw, int bh, double *tc, double *ts) {
    const int n = bw * bh;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            for (int jj = 0; jj < bh; jj++)
                for (int ii = 0; ii < bw; ii++) {
                    double ang = 2 * ORC_PHASE_PI * ((1.0 * i * ii / bw) + (1.0 * j * jj / bh));
                    tc[(j * bw + i) * n + jj * bw + ii] = cos(ang);
                    ts[(j * bw + i) * n + jj * bw + ii] = sin(ang);
                }
}

/* Normalised cross-power spectrum (:108-130), inverse DFT (:132-142) and
 * peak search (:144-157, first strict maximum above 0 in raster order,
 * 1-based coordinates). Returns sqrt(x^2 + y^2) of the peak as float, 0 when
 * no value is positive. */
static float orc_phase_peak(const double *rr, const double *ri, const double *cr, const double *ci, int bw,
                            int bh, const double *tc, const double *ts, double *xr, double *xi) {
    const int n = bw * bh;
    const double sn = sqrt((double)n);
    for (int i = 0; i < n; i++) {
        double conj = (-1) * ci[i];
        double multReal = rr[i] * cr[i] - ri[i] * conj;
        double multImag = rr[i] * conj + ri[i] * cr[i];
        double ar = fabs(multReal), ai = fabs(multImag);
        xr[i] = ((multReal * ar) + (multImag * ai)) / ((ar * ar) + (ai * ai) + ORC_EPS);
        xi[i] = ((multImag * ar) - (multReal * ai)) / ((ar * ar) + (ai * ai) + ORC_EPS);
    }
    double max_value = 0.0;
    int xc = 0, yc = 0;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++) {
            const int a = j * bw + i;
            double v = 0.0;
            for (int b = 0; b < n; b++) v += (xr[b] * tc[a * n + b] - xi[b] * ts[a * n + b]) / sn;
            if (v > max_value) {
                max_value = v;
                xc = i + 1;
                yc = j + 1;
            }
        }
    return (float)sqrt(((double)xc * (double)xc) + ((double)yc * (double)yc));
}

/* getExpDecayWeight of cl/kernelGetPhaseCorrelationMap.cl:167-179. */
static float orc_phase_weight(float ref, float comp) {
    float weight = 0;
    if (ref == comp) weight = 1;
    else weight = 1 - (2 * (fabsf(ref - comp) / (fabsf(ref) + fabsf(comp))));
    return weight;
}

/* Normalised whole-square patch of :46-57 / :80-91. */
static void orc_phase_patch(const float *img, const float *means, const float *stds, int W, int bw, int bh,
                            int x0, int y0, double *x) {
    const int rw = bw / 2, rh = bh / 2;
    int c = 0;
    for (int j = y0 - rh; j <= y0 + rh; j++)
        for (int i = x0 - rw; i <= x0 + rw; i++)
            x[c++] = ((double)img[j * W + i] - (double)means[y0 * W + x0]) /
                     ((double)stds[y0 * W + x0] + ORC_EPS);
}

/* cl/kernelGetPhaseCorrelationMap.cl:21-164 (repaired as stated above) for
 * every interior reference pixel. f64acc as in orc_hu_map. Returns -1 for a
 * block larger than 15 x 15. */
int orc_phase_map(const float *img, const float *means, const float *stds, int W, int H, int bw, int bh,
                  int f64acc, double *out) {
    const int rw = bw / 2, rh = bh / 2, n = bw * bh;
    if (n > 225) return -1;
    const int nx = W - 2 * rw, ny = H - 2 * rh;
    double *tc = (double *)malloc(sizeof(double) * n * n), *ts = (double *)malloc(sizeof(double) * n * n);
    double *fr = (double *)malloc(sizeof(double) * n * (size_t)nx * ny);
    double *fi = (double *)malloc(sizeof(double) * n * (size_t)nx * ny);
    orc_phase_tables(bw, bh, tc, ts);
    #pragma omp parallel for schedule(static)
    for (int y = rh; y < H - rh; y++)
        for (int xq = rw; xq < W - rw; xq++) {
            double x[225];
            const size_t b = (size_t)(y - rh) * nx + (xq - rw);
            orc_phase_patch(img, means, stds, W, bw, bh, xq, y, x);
            orc_phase_dft(x, n, tc, ts, fr + b * n, fi + b * n);
        }
    #pragma omp parallel for schedule(dynamic, 1)
    for (int y0 = rh; y0 < H - rh; y0++)
        for (int x0 = rw; x0 < W - rw; x0++) {
            double xr[225], xi[225];
            const size_t p = (size_t)(y0 - rh) * nx + (x0 - rw);
            float acc32 = 0.0f;
            double acc64 = 0.0;
            for (int y1 = rh; y1 < H - rh; y1++)
                for (int x1 = rw; x1 < W - rw; x1++) {
                    const size_t q = (size_t)(y1 - rh) * nx + (x1 - rw);
                    float d = orc_phase_peak(fr + p * n, fi + p * n, fr + q * n, fi + q * n, bw, bh, tc, ts, xr, xi);
                    double weight = (double)orc_phase_weight(stds[y0 * W + x0], stds[y1 * W + x1]);
                    acc32 = (float)((double)acc32 + (double)d * weight);
                    acc64 += (double)d * weight;
                }
            out[y0 * W + x0] = f64acc ? acc64 : (double)acc32;
        }
    free(tc); free(ts); free(fr); free(fi);
    return 0;
}

/* Block-map form of the phase correlation (a definition of this library, the
 * reference has only the all-pairs kernel): the reference block
 * (ReferenceBlock2D pixels / (std + eps)) and each interior block
 * ((x - mean) / (std + eps) with the block's FP32 local statistics), both on
 * the ellipse and 0 elsewhere on the bw x bh grid, go through the exact DFT
 * (twiddles cos / sin(2 pi m / L), m = (a b) mod L; direct sums, rows then
 * columns), the kernel's normalised cross-power spectrum (:108-130), the real
 * part of the exact inverse DFT (rows, then columns) divided by
 * sqrt(bw bh), and the kernel's peak search (:144-157: first strict maximum
 * above 0 in raster order, 1-based coordinates); out = peak distance. */
static void orc_exact_tables(int L, double *c, double *s) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < L; m++) {
        c[m] = cos(two_pi * m / L);
        s[m] = sin(two_pi * m / L);
    }
}

static void orc_exact_dft(const double *x, int bw, int bh, const double *cw, const double *sw, const double *ch,
                          const double *sh, double *re, double *im) {
    double tr[225], ti[225];
    for (int jj = 0; jj < bh; jj++)
        for (int i = 0; i < bw; i++) {
            double sr = 0.0, si = 0.0;
            for (int ii = 0; ii < bw; ii++) {
                const int m = (i * ii) % bw;
                sr += x[jj * bw + ii] * cw[m];
                si -= x[jj * bw + ii] * sw[m];
            }
            tr[jj * bw + i] = sr;
            ti[jj * bw + i] = si;
        }
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++) {
            double sr = 0.0, si = 0.0;
            for (int jj = 0; jj < bh; jj++) {
                const int m = (j * jj) % bh;
                sr += tr[jj * bw + i] * ch[m] + ti[jj * bw + i] * sh[m];
                si += ti[jj * bw + i] * ch[m] - tr[jj * bw + i] * sh[m];
            }
            re[j * bw + i] = sr;
            im[j * bw + i] = si;
        }
}

int orc_block_phase(const float *img, const float *means, const float *stds, int W, int H, int bw, int bh,
                    const float *ref_pixels, float ref_std, double *out) {
    const int rw = bw / 2, rh = bh / 2, n = bw * bh;
    if (bw > 15 || bh > 15) return -1;
    double cw[15], sw[15], ch[15], sh[15];
    orc_exact_tables(bw, cw, sw);
    orc_exact_tables(bh, ch, sh);
    double x[225], rr[225], ri[225];
    int k = 0;
    for (int j = 0; j < bh; j++)
        for (int i = 0; i < bw; i++)
            x[j * bw + i] = in_ellipse(i - rw, j - rh, rw, rh)
                                ? (double)ref_pixels[k++] / ((double)ref_std + ORC_EPS) : 0.0;
    orc_exact_dft(x, bw, bh, cw, sw, ch, sh, rr, ri);
    const double sn = sqrt((double)n);
    #pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; y++)
        for (int xq = 0; xq < W; xq++) {
            double xv[225], cr[225], ci[225], xr[225], xi[225], sr_[225], si_[225];
            if (xq < rw || xq >= W - rw || y < rh || y >= H - rh) {
                out[y * W + xq] = 0.0;
                continue;
            }
            const double m = (double)means[y * W + xq], s = (double)stds[y * W + xq] + ORC_EPS;
            for (int j = 0; j < bh; j++)
                for (int i = 0; i < bw; i++)
                    xv[j * bw + i] = in_ellipse(i - rw, j - rh, rw, rh)
                                         ? ((double)img[(y + j - rh) * W + xq + i - rw] - m) / s : 0.0;
            orc_exact_dft(xv, bw, bh, cw, sw, ch, sh, cr, ci);
            for (int i = 0; i < n; i++) {
                double conj = (-1) * (ci[i] / sn), q = cr[i] / sn;
                double multReal = rr[i] * q - ri[i] * conj;
                double multImag = rr[i] * conj + ri[i] * q;
                double ar = fabs(multReal), ai = fabs(multImag);
                xr[i] = ((multReal * ar) + (multImag * ai)) / ((ar * ar) + (ai * ai) + ORC_EPS);
                xi[i] = ((multImag * ar) - (multReal * ai)) / ((ar * ar) + (ai * ai) + ORC_EPS);
            }
            /* inverse: rows, then the real part over columns */
            for (int jj = 0; jj < bh; jj++)
                for (int i = 0; i < bw; i++) {
                    double a = 0.0, b = 0.0;
                    for (int ii = 0; ii < bw; ii++) {
                        const int mm = (i * ii) % bw;
                        a += xr[jj * bw + ii] * cw[mm] - xi[jj * bw + ii] * sw[mm];
                        b += xr[jj * bw + ii] * sw[mm] + xi[jj * bw + ii] * cw[mm];
                    }
                    sr_[jj * bw + i] = a;
                    si_[jj * bw + i] = b;
                }
            double max_value = 0.0;
            int xc = 0, yc = 0;
            for (int j = 0; j < bh; j++)
                for (int i = 0; i < bw; i++) {
                    double v = 0.0;
                    for (int jj = 0; jj < bh; jj++) {
                        const int mm = (j * jj) % bh;
                        v += sr_[jj * bw + i] * ch[mm] - si_[jj * bw + i] * sh[mm];
                    }
                    v /= sn;
                    if (v > max_value) {
                        max_value = v;
                        xc = i + 1;
                        yc = j + 1;
                    }
                }
            out[y * W + xq] = (double)(float)sqrt(((double)xc * (double)xc) + ((double)yc * (double)yc));
        }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Variance stabilisation (generalised Anscombe transform)             */
/* ------------------------------------------------------------------ */

/* java/VarianceStabilisingTransform2D_.java:136-151 (getGAT), in place. */
void orc_gat(float *img, int n, double gain, double sigma, double offset) {
    double refConstant = (3.0 / 8.0) * gain * gain + sigma * sigma - gain * offset;
    for (int i = 0; i < n; i++) {
        double v = (double)img[i];
        if ((gain * v + refConstant) < 0.0) v = 0.0;
        else v = (2.0 / gain) * sqrt(gain * v + refConstant);
        img[i] = (float)v;
    }
}

/* java/GATMinimizer2D.java userFunction with applyGAT and getMeanAndVarBlock:
 * width/6 x height/6 blocks, sum of (variance - 1)^2 / blocks. Returns -1 when
 * the grid has fewer than 2 blocks a side. */
double orc_gat_objective(const float *pixels, int width, int height, double gain, double sigma, double offset) {
    double refConstant = (3.0 / 8.0) * gain * gain + sigma * sigma - gain * offset;
    int blockWidth = width / 6, blockHeight = height / 6;
    if (blockWidth < 1 || blockHeight < 1) return -1.0;
    int nBlocksX = width / blockWidth, nBlocksY = height / blockHeight;
    if (nBlocksX < 2 || nBlocksY < 2) return -1.0;
    float *g = (float *)malloc(sizeof(float) * (size_t)width * height);
    for (int n = 0; n < width * height; n++) {
        double v = pixels[n];
        if (v <= -refConstant / gain) v = 0;
        else v = (2 / gain) * sqrt(gain * v + refConstant);
        g[n] = (float)v;
    }
    int nBlocks = nBlocksX * nBlocksY;
    double error = 0;
    for (int bY = 0; bY < nBlocksY; bY++)
        for (int bX = 0; bX < nBlocksX; bX++) {
            double mean = 0, sq_sum = 0;
            int bWH = blockWidth * blockHeight;
            for (int j = bY * blockHeight; j < (bY + 1) * blockHeight; j++)
                for (int i = bX * blockWidth; i < (bX + 1) * blockWidth; i++) {
                    float v = g[j * width + i];
                    mean += v;
                    sq_sum += v * v;
                }
            mean = mean / bWH;
            double var = sq_sum / bWH - mean * mean;
            double delta = var - 1;
            error += (delta * delta) / (double)nBlocks;
        }
    free(g);
    return error;
}

/* ------------------------------------------------------------------ */
/* 3D block repetition maps                                            */
/* ------------------------------------------------------------------ */

/* Inscribed-ellipsoid test of the 3D code (java/Utils.java:1075-1085,
 * cl/kernelGetLocalStatistics3D.cl:35-38), float arithmetic, same order. */
static int in_ellipsoid(int dx, int dy, int dz, int rw, int rh, int rd) {
    float fx = (float)dx, fy = (float)dy, fz = (float)dz;
    return ((fx * fx) / (float)(rw * rw)) + ((fy * fy) / (float)(rh * rh)) + ((fz * fz) / (float)(rd * rd)) <= 1.0f;
}

int orc_block_size3d(int bw, int bh, int bd) {
    int rw = bw / 2, rh = bh / 2, rd = bd / 2, k = 0;
    for (int z = -rd; z <= rd; z++)
        for (int y = -rh; y <= rh; y++)
            for (int x = -rw; x <= rw; x++) k += in_ellipsoid(x, y, z, rw, rh, rd);
    return k;
}

/* Linear offsets of the ellipsoid in raster order (z, y, x). */
static int ellipsoid_offsets(int bw, int bh, int bd, int W, int H, long *off) {
    int rw = bw / 2, rh = bh / 2, rd = bd / 2, k = 0;
    for (int z = -rd; z <= rd; z++)
        for (int y = -rh; y <= rh; y++)
            for (int x = -rw; x <= rw; x++)
                if (in_ellipsoid(x, y, z, rw, rh, rd)) off[k++] = (long)z * W * H + (long)y * W + x;
    return k;
}

static int interior3d(int x, int y, int z, int W, int H, int D, int rw, int rh, int rd) {
    return x >= rw && x < W - rw && y >= rh && y < H - rh && z >= rd && z < D - rd;
}

/* cl/kernelGetLocalStatistics3D.cl:11-61 for every voxel. */
void orc_local_stats3d_f32(const float *img, int W, int H, int D, int bw, int bh, int bd, float *means,
                           float *stds) {
    const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
    long off[4096];
    const int K = ellipsoid_offsets(bw, bh, bd, W, H, off);
    #pragma omp parallel for schedule(static)
    for (int z = 0; z < D; z++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const long p = (long)z * W * H + (long)y * W + x;
                if (!interior3d(x, y, z, W, H, D, rw, rh, rd)) {
                    means[p] = 0.0f;
                    stds[p] = 0.0f;
                    continue;
                }
                float mean = 0.0f;
                for (int i = 0; i < K; i++) mean += img[p + off[i]];
                mean /= (float)K;
                float var = 0.0f;
                for (int i = 0; i < K; i++) var += (img[p + off[i]] - mean) * (img[p + off[i]] - mean);
                means[p] = mean;
                stds[p] = sqrtf(var / (float)(K - 1));
            }
}

/* java/Utils.java:1642-1662 (normalizeArray). */
static void orc_normalize_array(float *a, int n) {
    float mn = 3.40282347e38f, mx = -3.40282347e38f;
    for (int i = 0; i < n; i++) {
        mn = jmin(a[i], mn);
        mx = jmax(a[i], mx);
    }
    for (int i = 0; i < n; i++) a[i] = (a[i] - mn) / (mx - mn + ORC_EPS);
}

/* java/Utils.java:1047-1160 (getReferenceBlock3D) for a block given as
 * bd slices of bh x bw floats: ellipsoid-flatten, normalise, subtract the
 * mean, normalise again; mean and (K-1) std of the result. Returns K. */
int orc_reference_block3d(const float *blk, int bw, int bh, int bd, float *pixels, float *mean_out,
                          float *std_out) {
    const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
    int K = 0;
    for (int z = 0; z < bd; z++)
        for (int y = 0; y < bh; y++)
            for (int x = 0; x < bw; x++)
                if (in_ellipsoid(x - rw, y - rh, z - rd, rw, rh, rd)) pixels[K++] = blk[(z * bh + y) * bw + x];
    orc_normalize_array(pixels, K);
    float m = 0.0f;
    for (int i = 0; i < K; i++) m += pixels[i];
    m /= (float)K;
    for (int i = 0; i < K; i++) pixels[i] = pixels[i] - m;
    orc_normalize_array(pixels, K);
    m = 0.0f;
    for (int i = 0; i < K; i++) m += pixels[i];
    m /= (float)K;
    float s = 0.0f;
    for (int i = 0; i < K; i++) s += (pixels[i] - m) * (pixels[i] - m);
    *mean_out = m;
    *std_out = (float)sqrt((double)(s / ((float)(K - 1))));
    return K;
}

/* cl/kernelGetBlock{Pearson,Ssim,Nrmse,AbsDiffStds}3D.cl for every voxel,
 * with the block radii of the block itself (the reference's Pearson command
 * passes the block depth as the z radius, java/CLUtils.java:1149; repaired). */
void orc_block3d_kernel_f32(int metric, const float *img, int W, int H, int D, int bw, int bh, int bd,
                            const float *means, const float *stds, const float *ref, int K, float ref_mean,
                            float ref_std, float *out) {
    const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
    long off[4096];
    ellipsoid_offsets(bw, bh, bd, W, H, off);
    #pragma omp parallel for schedule(static)
    for (int z = 0; z < D; z++)
        for (int y = 0; y < H; y++)
            for (int x = 0; x < W; x++) {
                const long p = (long)z * W * H + (long)y * W + x;
                if (!interior3d(x, y, z, W, H, D, rw, rh, rd)) {
                    out[p] = 0.0f;
                    continue;
                }
                float t[4096];
                const float tstd = stds[p], tmean = means[p];
                if (metric == ORC_ABSDIFF) {
                    out[p] = fabsf((float)ref_std - (float)tstd);
                    continue;
                }
                for (int i = 0; i < K; i++) t[i] = img[p + off[i]];
                if (metric == ORC_PEARSON) {
                    float mn = FLT_MAX, mx = -FLT_MAX;
                    for (int i = 0; i < K; i++) {
                        mn = fminf(mn, t[i]);
                        mx = fmaxf(mx, t[i]);
                    }
                    for (int i = 0; i < K; i++) t[i] = (t[i] - mn) / (mx - mn + ORC_EPS);
                    for (int i = 0; i < K; i++) t[i] = t[i] - tmean;
                    mn = FLT_MAX;
                    mx = -FLT_MAX;
                    for (int i = 0; i < K; i++) {
                        mn = fminf(mn, t[i]);
                        mx = fmaxf(mx, t[i]);
                    }
                    for (int i = 0; i < K; i++) t[i] = (t[i] - mn) / (mx - mn + ORC_EPS);
                    float cov = 0.0f;
                    for (int i = 0; i < K; i++) cov += ref[i] * t[i];
                    cov /= (float)(K - 1);
                    if (ref_std == 0.0 && tstd == 0.0) out[p] = 1.0f;
                    else if (ref_std == 0.0 || tstd == 0.0) out[p] = 0.0f;
                    else out[p] = fmaxf(0.0f, (float)(cov / ((ref_std * tstd) + ORC_EPS)));
                } else if (metric == ORC_SSIM) {
                    for (int i = 0; i < K; i++) t[i] = t[i] - tmean;
                    float cov = 0.0f;
                    for (int i = 0; i < K; i++) cov += ref[i] * t[i];
                    cov /= (float)(K - 1);
                    const float c1 = 0.0001f, c2 = 0.0009f;
                    if (ref_std == 0.0 && tstd == 0.0) out[p] = 1.0f;
                    else if (ref_std == 0.0 || tstd == 0.0) out[p] = 0.0f;
                    else {
                        float ssim = (float)((2.0f * ref_mean * tmean + c1) * (2.0f * cov + c2)) /
                                     (((ref_mean * ref_mean) + (tmean * tmean) + c1) *
                                      ((ref_std * ref_std) + (tstd * tstd) + c2));
                        out[p] = fmaxf(0.0f, ssim);
                    }
                } else { /* NRMSE */
                    for (int i = 0; i < K; i++) t[i] = t[i] - tmean;
                    float mse = 0.0f;
                    for (int i = 0; i < K; i++) mse += (ref[i] - t[i]) * (ref[i] - t[i]);
                    mse /= (float)K;
                    out[p] = sqrtf(mse);
                }
            }
}

/* java/Utils.java:1463-1498 (getMeanNoiseVar3D from local stds): the mean
 * local variance over the interior, FP32, raster order; the element count is
 * a float (it stops growing at 2^24). */
float orc_noise_var3d(int W, int H, int D, int rw, int rh, int rd, const float *stds) {
    float s = 0.0f, n = 0.0f;
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                long i = (long)W * H * z + (long)y * W + x;
                s += stds[i] * stds[i];
                n += 1.0f;
            }
    return s / n;
}

/* java/Utils.java:1501-1525 (getRelevanceMask3D). Returns the noise variance. */
float orc_relevance_mask3d(int W, int H, int D, int rw, int rh, int rd, const float *stds, float c, float *mask) {
    const float nv = orc_noise_var3d(W, H, D, rw, rh, rd, stds);
    memset(mask, 0, sizeof(float) * (size_t)W * H * D);
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                long i = (long)W * H * z + (long)y * W + x;
                mask[i] = (stds[i] * stds[i]) <= nv * c ? 0.0f : 1.0f;
            }
    return nv;
}

/* java/Utils.java:1572-1630 (normalizeImage3D), in place; mask may be NULL. */
void orc_normalize_image3d(float *a, int W, int H, int D, int rw, int rh, int rd, const float *mask) {
    float mn = 3.40282347e38f, mx = -3.40282347e38f;
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                long i = (long)W * H * z + (long)y * W + x;
                if (!mask || mask[i] > 0.0f) {
                    mn = jmin(a[i], mn);
                    mx = jmax(a[i], mx);
                }
            }
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                long i = (long)W * H * z + (long)y * W + x;
                if (!mask || mask[i] > 0.0f) a[i] = (a[i] - mn) / (mx - mn + ORC_EPS);
            }
}

/* Host steps after the 3D block kernels (java/CLUtils.java:1133-1637): NRMSE
 * inverted (0 -> 1) and Abs-diff turned into 1 - x over the interior, the
 * relevance mask applied when c > 0, normalisation over the interior (over
 * the mask when c > 0). */
void orc_block3d_postprocess_f32(int metric, float *map, int W, int H, int D, int rw, int rh, int rd,
                                 const float *stds, float c, int normalize) {
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                long i = (long)W * H * z + (long)y * W + x;
                if (metric == ORC_NRMSE) map[i] = map[i] == 0.0f ? 1.0f : 1.0f / map[i];
                else if (metric == ORC_ABSDIFF) map[i] = 1.0f - map[i];
            }
    float *mask = NULL;
    if (c > 0.0f) {
        mask = (float *)malloc(sizeof(float) * (size_t)W * H * D);
        orc_relevance_mask3d(W, H, D, rw, rh, rd, stds, c, mask);
        for (long i = 0; i < (long)W * H * D; i++) map[i] *= mask[i];
    }
    if (normalize) orc_normalize_image3d(map, W, H, D, rw, rh, rd, mask);
    free(mask);
}

/* ------------------------------------------------------------------ */
/* 3D global repetition maps                                           */
/* ------------------------------------------------------------------ */

/* cl/kernelGetGlobal{Pearson,Ssim,Nrmse,AbsDiffStds}3D.cl, FP32 in the kernels'
 * order, for the reference voxels listed in pix (num/den indexed like pix).
 * Differences from the 2D kernels that these kernels carry: a reference voxel
 * with zero local variance is skipped (:37), NRMSE accumulates sqrt(mse) times
 * the weight, Abs-diff skips test voxels of zero variance. Two defects are
 * repaired: the reference block is gathered over z <= gz + bRZ (the kernels
 * stop at z < gz + bRZ, :46, leaving the last slice's ellipsoid voxels at 0
 * before the mean subtraction), and SSIM's below-threshold branch adds to its
 * own map (kernelGetGlobalSsim3D.cl:76 names an undeclared pearson_map and
 * does not compile). */
void orc_global3d_f32(int metric, const float *img, int W, int H, int D, int bw, int bh, int bd,
                      const float *means, const float *stds, float filter_param, float threshold,
                      const int *pix, int n_pix, float *num, float *den) {
    const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
    long *off = (long *)malloc(sizeof(long) * bw * bh * bd);
    const int K = ellipsoid_offsets(bw, bh, bd, W, H, off);
    const float c1 = 0.0001f, c2 = 0.0009f;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int ii = 0; ii < n_pix; ii++) {
        const long p = pix[ii];
        const int gx = (int)(p % W), gy = (int)((p / W) % H), gz = (int)(p / ((long)W * H));
        float S = 0.0f, Wsum = 0.0f;
        float rb[4096], tb[4096];
        num[ii] = 0.0f;
        den[ii] = 0.0f;
        if (!interior3d(gx, gy, gz, W, H, D, rw, rh, rd)) continue;
        const float rs = stds[p];
        const float rv = rs * rs;
        if (rv < threshold || rv == 0.0f) continue;
        const float rm = means[p];
        if (metric != ORC_ABSDIFF)
            for (int i = 0; i < K; i++) rb[i] = img[p + off[i]] - rm;
        for (int z = rd; z < D - rd; z++)
            for (int y = rh; y < H - rh; y++)
                for (int x = rw; x < W - rw; x++) {
                    const long q = (long)W * H * z + (long)y * W + x;
                    const float ts = stds[q];
                    const float tv = ts * ts;
                    if (tv < threshold) continue;
                    if (metric == ORC_ABSDIFF) {
                        if (tv == 0.0f) continue;
                        const float wgt = expf((-1.0f) * (((rs - ts) * (rs - ts)) / (filter_param + ORC_EPS)));
                        Wsum += wgt;
                        S += fmaxf(0.0f, fabsf(rs - ts)) * wgt;
                        continue;
                    }
                    const float tm = means[q];
                    for (int i = 0; i < K; i++) tb[i] = img[q + off[i]] - tm;
                    const float wgt = expf((-1.0f) * (((rs - ts) * (rs - ts)) / (filter_param + ORC_EPS)));
                    if (metric == ORC_NRMSE) {
                        Wsum += wgt;
                        float mse = 0.0f;
                        for (int i = 0; i < K; i++) mse += (rb[i] - tb[i]) * (rb[i] - tb[i]);
                        mse /= (float)K;
                        S += sqrtf(mse) * wgt;
                        continue;
                    }
                    float cov = 0.0f;
                    for (int i = 0; i < K; i++) cov += rb[i] * tb[i];
                    cov /= (float)(K - 1);
                    Wsum += wgt;
                    if (ts == 0.0f) {
                        S += 0.0f;
                    } else if (metric == ORC_PEARSON) {
                        S += fmaxf(0.0f, cov / ((rs * ts) + ORC_EPS)) * wgt;
                    } else {
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

/* The same sums in FP64 (the judge): block moments and vectors in FP64 from
 * the FP32 voxels; relevance and flatness decisions on the FP32 stds. */
void orc_global3d_f64(int metric, const float *img, int W, int H, int D, int bw, int bh, int bd,
                      const float *stds32, float filter_param, float threshold, const int *pix, int n_pix,
                      double *num, double *den) {
    const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
    long *off = (long *)malloc(sizeof(long) * bw * bh * bd);
    const int K = ellipsoid_offsets(bw, bh, bd, W, H, off);
    long nint = (long)(W - 2 * rw > 0 ? W - 2 * rw : 0) * (H - 2 * rh > 0 ? H - 2 * rh : 0) *
                (D - 2 * rd > 0 ? D - 2 * rd : 0);
    long nq = 0;
    long *qi = (long *)malloc(sizeof(long) * (size_t)(nint > 0 ? nint : 1));
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                const long q = (long)W * H * z + (long)y * W + x;
                const float s = stds32[q];
                if (s * s < threshold) continue;
                if (metric == ORC_ABSDIFF && s * s == 0.0f) continue;
                qi[nq++] = q;
            }
    double *qv = (double *)malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1) * K);
    double *qm = (double *)malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1));
    double *qs = (double *)malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1));
    #pragma omp parallel for schedule(static)
    for (long j = 0; j < nq; j++) {
        const long q = qi[j];
        double m = 0.0, v = 0.0;
        for (int i = 0; i < K; i++) m += (double)img[q + off[i]];
        m /= K;
        for (int i = 0; i < K; i++) {
            const double d = (double)img[q + off[i]] - m;
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
        const long p = pix[ii];
        const int gx = (int)(p % W), gy = (int)((p / W) % H), gz = (int)(p / ((long)W * H));
        num[ii] = 0;
        den[ii] = 0;
        if (!interior3d(gx, gy, gz, W, H, D, rw, rh, rd)) continue;
        const float rs32 = stds32[p];
        if (rs32 * rs32 < threshold || rs32 * rs32 == 0.0f) continue;
        double rb[4096], rm = 0.0, rv = 0.0;
        for (int i = 0; i < K; i++) rm += (double)img[p + off[i]];
        rm /= K;
        for (int i = 0; i < K; i++) {
            rb[i] = (double)img[p + off[i]] - rm;
            rv += rb[i] * rb[i];
        }
        const double rs = sqrt(rv / (K - 1));
        double S = 0.0, Ws = 0.0;
        for (long j = 0; j < nq; j++) {
            const double *tb = qv + (size_t)j * K;
            const double ts = qs[j], tm = qm[j];
            const double wgt = exp(-((rs - ts) * (rs - ts)) / h);
            Ws += wgt;
            if (metric == ORC_ABSDIFF) {
                S += fabs(rs - ts) * wgt;
                continue;
            }
            if (metric == ORC_NRMSE) {
                double mse = 0.0;
                for (int i = 0; i < K; i++) {
                    const double d = rb[i] - tb[i];
                    mse += d * d;
                }
                S += sqrt(mse / K) * wgt;
                continue;
            }
            if (stds32[qi[j]] == 0.0f) continue;
            double cov = 0.0;
            for (int i = 0; i < K; i++) cov += rb[i] * tb[i];
            cov /= (K - 1);
            if (metric == ORC_PEARSON) {
                const double r = cov / (rs * ts + (double)ORC_EPS);
                S += (r > 0.0 ? r : 0.0) * wgt;
            } else {
                const double s = ((2.0 * rm * tm + c1) * (2.0 * cov + c2)) /
                                 ((rm * rm * tm * tm + c1) * (rs * rs + ts * ts + c2)) * wgt;
                S += s > 0.0 ? s : 0.0;
            }
        }
        num[ii] = S;
        den[ii] = Ws;
    }
    free(off);
    free(qi);
    free(qv);
    free(qm);
    free(qs);
}

/* nPixels of the 3D command (java/GlobalRepetition3D_.java:132-143): 1.0f per
 * interior voxel with mask > 0, summed in FP32. */
float orc_n_pixels3d(const float *mask, int W, int H, int D, int rw, int rh, int rd) {
    float n = 0.0f;
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++)
                if (mask[(long)W * H * z + (long)y * W + x] > 0.0f) n += 1.0f;
    return n;
}

/* Host steps of getGlobal*3D (java/CLUtils.java:2225-2790) on a full W*H*D
 * map of num/den: num / (den * nPixels + eps) over the interior; NRMSE and
 * Abs-diff inverted where mask > 0 (0 -> 1); the mask applied when the
 * relevance constant is > 0; normalizeImage3D over the mask (always given). */
void orc_global3d_finalize_f32(int metric, const float *num, const float *den, int W, int H, int D, int rw,
                               int rh, int rd, const float *mask, float relevance_constant, float n_pixels,
                               int normalize, float *out) {
    const long n = (long)W * H * D;
    memset(out, 0, sizeof(float) * (size_t)n);
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                const long i = (long)W * H * z + (long)y * W + x;
                out[i] = num[i] / (den[i] * n_pixels + ORC_EPS);
            }
    if (metric == ORC_NRMSE || metric == ORC_ABSDIFF)
        for (int z = rd; z < D - rd; z++)
            for (int y = rh; y < H - rh; y++)
                for (int x = rw; x < W - rw; x++) {
                    const long i = (long)W * H * z + (long)y * W + x;
                    if (mask[i] > 0.0f) out[i] = (out[i] == 0.0f) ? 1.0f : 1.0f / out[i];
                }
    if (relevance_constant > 0.0f)
        for (long i = 0; i < n; i++) out[i] *= mask[i];
    if (normalize) orc_normalize_image3d(out, W, H, D, rw, rh, rd, mask);
}

/* The same steps in FP64 on FP64 sums (the judge's map). */
void orc_global3d_finalize_f64(int metric, const double *num, const double *den, int W, int H, int D, int rw,
                               int rh, int rd, const float *mask, float relevance_constant, double n_pixels,
                               int normalize, double *out) {
    const long n = (long)W * H * D;
    memset(out, 0, sizeof(double) * (size_t)n);
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                const long i = (long)W * H * z + (long)y * W + x;
                out[i] = num[i] / (den[i] * n_pixels + (double)ORC_EPS);
                if ((metric == ORC_NRMSE || metric == ORC_ABSDIFF) && mask[i] > 0.0f)
                    out[i] = (out[i] == 0.0) ? 1.0 : 1.0 / out[i];
            }
    if (relevance_constant > 0.0f)
        for (long i = 0; i < n; i++) out[i] *= (double)mask[i];
    if (!normalize) return;
    double mn = DBL_MAX, mx = -DBL_MAX;
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                const long i = (long)W * H * z + (long)y * W + x;
                if (!(mask[i] > 0.0f)) continue;
                if (out[i] < mn) mn = out[i];
                if (out[i] > mx) mx = out[i];
            }
    for (int z = rd; z < D - rd; z++)
        for (int y = rh; y < H - rh; y++)
            for (int x = rw; x < W - rw; x++) {
                const long i = (long)W * H * z + (long)y * W + x;
                if (mask[i] > 0.0f) out[i] = (out[i] - mn) / (mx - mn + (double)ORC_EPS);
            }
}

/* ------------------------------------------------------------------ */
/* Relevance-mask tools (java/RelevanceMask2D_.java,                    */
/* java/RelevanceMaskStack2D_.java, java/OptimiseRelevanceMask_.java)   */
/* ------------------------------------------------------------------ */

/* cl/kernelGetRelevanceMask2D.cl (take_sqrt = 0: the local variance) and
 * cl/kernelGetLocalMeans.cl (take_sqrt = 1: its square root) over the ellipse
 * of a bw x bh block; border pixels 0 (the commands' buffers start at 0). */
void orc_local_var2d(const float *img, int W, int H, int bw, int bh, int take_sqrt, float *out) {
    const int rw = bw / 2, rh = bh / 2;
    int *off = (int *)malloc(sizeof(int) * bw * bh);
    const int K = ellipse_offsets(bw, bh, W, off);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const int p = y * W + x;
            if (x < rw || x >= W - rw || y < rh || y >= H - rh) { out[p] = 0.0f; continue; }
            float mean = 0.0f;
            for (int i = 0; i < K; i++) mean += img[p + off[i]];
            mean /= (float)K;
            float var = 0.0f;
            for (int i = 0; i < K; i++) var += (img[p + off[i]] - mean) * (img[p + off[i]] - mean);
            var /= (float)(K - 1);
            out[p] = take_sqrt ? sqrtf(var) : var;
        }
    free(off);
}

/* The tools' noise variance: tile variances with FP32 sums
 * (OptimiseRelevanceMask_.getMeanAndVarBlock, fp64 = 0) or FP64 sums
 * (RelevanceMask2D_.getMeanAndVarBlock, fp64 = 1), sorted, the lowest 3%
 * averaged in FP32, then (1 + 0.001 (v - 40)) v. Returns -1 if the image has
 * no tile. */
int orc_tool_noise_var(const float *img, int W, int H, int fp64, float *out) {
    const int wh = W * H, t = (wh <= 352 * 288) ? 8 : 16;
    const int nbx = W / t, nby = H / t, nb = nbx * nby;
    const int nv = (int)(0.03f * (float)nb + 1.0f);
    if (nv > nb) return -1;
    float *vars = (float *)malloc(sizeof(float) * (nb > 0 ? nb : 1));
    for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
            float var;
            if (fp64) {
                double mean = 0.0, sq = 0.0;
                for (int y = by * t; y < (by + 1) * t; y++)
                    for (int x = bx * t; x < (bx + 1) * t; x++) {
                        const float v = img[y * W + x];
                        mean += (double)v;
                        sq += (double)(v * v);
                    }
                mean = mean / (t * t);
                var = (float)(sq / (t * t) - mean * mean);
            } else {
                float mean = 0.0f, sq = 0.0f;
                for (int y = by * t; y < (by + 1) * t; y++)
                    for (int x = bx * t; x < (bx + 1) * t; x++) {
                        const float v = img[y * W + x];
                        mean += v;
                        sq += v * v;
                    }
                mean = mean / (float)(t * t);
                var = sq / (float)(t * t) - mean * mean;
            }
            vars[by * nbx + bx] = var;
        }
    qsort(vars, nb, sizeof(float), cmp_float);
    float v = 0.0f;
    for (int i = 0; i < nv; i++) v += vars[i];
    v = fabsf(v / (float)nv);
    *out = (1.0f + 0.001f * (v - 40.0f)) * v;
    free(vars);
    return 0;
}

/* OptimiseRelevanceMask_.getRelevanceMap's mask (also RelevanceMask2D_'s): an
 * interior pixel is 1 unless s^2 < threshold or s^2 == 0; threshold = nv * c,
 * or c when nv == 0. */
void orc_tool_mask(const float *stat, int W, int H, int rw, int rh, float nv, float c, float *mask) {
    const float thr = nv == 0.0f ? c : nv * c;
    memset(mask, 0, sizeof(float) * (size_t)W * H);
    for (int y = rh; y < H - rh; y++)
        for (int x = rw; x < W - rw; x++) {
            const float v = stat[y * W + x] * stat[y * W + x];
            mask[y * W + x] = (v < thr || v == 0.0f) ? 0.0f : 1.0f;
        }
}

/* OptimiseRelevanceMask_.run's loop, literally: whole masks at c = 0, step,
 * ... until one is all 0. Returns -1 if the constant stops increasing (the
 * reference would loop forever) or after max_iter masks. */
int orc_tool_range(const float *stat, int W, int H, int rw, int rh, float nv, float step, int max_iter,
                   float *all_ones, float *all_zeros) {
    float *m = (float *)malloc(sizeof(float) * (size_t)W * H);
    float fc = 0.0f, ones = 0.0f;
    int it = 0, rc = -1;
    for (; it < max_iter; it++) {
        orc_tool_mask(stat, W, H, rw, rh, nv, fc, m);
        int all1 = 1, all0 = 1;
        for (int y = rh; y < H - rh && all1; y++)
            for (int x = rw; x < W - rw; x++)
                if (m[y * W + x] != 1.0f) { all1 = 0; break; }
        for (int i = 0; i < W * H; i++)
            if (m[i] != 0.0f) { all0 = 0; break; }
        if (all1) ones = fc;
        if (all0) { rc = 0; break; }
        const float next = fc + step;
        if (!(next > fc)) break;
        fc = next;
    }
    free(m);
    *all_ones = ones;
    *all_zeros = fc;
    return rc;
}

/* ------------------------------------------------------------------ */
/* 3D variance stabilisation objective (java/GATMinimizer3D.java        */
/* userFunction, java/Utils.java getMeanAndVarBlock3D), sequential FP64 */
/* ------------------------------------------------------------------ */
double orc_gat_objective3d(const float *vox, int W, int H, int D, double gain, double sigma, double offset) {
    if (gain <= 0 || sigma < 0 || offset < 0) return NAN;
    const long n = (long)W * H * D;
    float *g = (float *)malloc(sizeof(float) * (size_t)n);
    const double c = (3.0 / 8.0) * gain * gain + sigma * sigma - gain * offset;
    for (long i = 0; i < n; i++) {
        double v = vox[i];
        v = (v <= -c / gain) ? 0.0 : (2 / gain) * sqrt(gain * v + c);
        g[i] = (float)v;
    }
    int bw = W / 6 > 1 ? W / 6 : 1, bh = H / 6 > 1 ? H / 6 : 1, bd = D / 6 > 1 ? D / 6 : 1;
    int nx = W / bw, ny = H / bh, nz = D / bd;
    while (nx < 2 || ny < 2 || nz < 2) {
        const int a0 = bw, b0 = bh, c0 = bd;
        if (nx < 2 && bw > 1) bw = bw / 2 > 1 ? bw / 2 : 1;
        if (ny < 2 && bh > 1) bh = bh / 2 > 1 ? bh / 2 : 1;
        if (nz < 2 && bd > 1) bd = bd / 2 > 1 ? bd / 2 : 1;
        nx = W / bw;
        ny = H / bh;
        nz = D / bd;
        if (bw == 1 && bh == 1 && bd == 1) break;
        if (bw == a0 && bh == b0 && bd == c0) break; /* an axis of 1 voxel: the reference loops forever */
    }
    const int nb = nx * ny * nz;
    double error = 0.0;
    for (int bz = 0; bz < nz; bz++)
        for (int by = 0; by < ny; by++)
            for (int bx = 0; bx < nx; bx++) {
                double mean = 0.0, sq = 0.0;
                for (int z = bz * bd; z < (bz + 1) * bd; z++)
                    for (int y = by * bh; y < (by + 1) * bh; y++)
                        for (int x = bx * bw; x < (bx + 1) * bw; x++) {
                            const double v = (double)g[(long)W * H * z + (long)y * W + x];
                            mean += v;
                            sq += v * v;
                        }
                const int bs = bw * bh * bd;
                mean = mean / bs;
                const double var = sq / bs - mean * mean;
                const double delta = var - 1.0;
                error += (delta * delta) / (double)nb;
            }
    free(g);
    return error;
}

/* ------------------------------------------------------------------ */
/* Redundancy classification (java/ClassifyRedundancy_.java): k-means++ */
/* and Lloyd as commons-math3 3.6.1 KMeansPlusPlusClusterer runs them,  */
/* with java.util.Random, and every sum in the library's fixed block     */
/* order (blocks of 1024 points; thread t of 256 adds points t, t + 256, */
/* t + 512, t + 768 of its block; then pairwise t += t + 128 ... t + 1;   */
/* blocks added in turn).                                                */
/* ------------------------------------------------------------------ */
#define KM_T 256
#define KM_PER 4
#define KM_SPAN (KM_T * KM_PER)

typedef struct { uint64_t seed; } jrand;
static void jr_init(jrand *r, int64_t s) { r->seed = ((uint64_t)s ^ 0x5DEECE66DULL) & ((1ULL << 48) - 1); }
static int jr_next(jrand *r, int bits) {
    r->seed = (r->seed * 0x5DEECE66DULL + 0xBULL) & ((1ULL << 48) - 1);
    return (int)(int64_t)(r->seed >> (48 - bits));
}
static int jr_int(jrand *r, int bound) {
    if ((bound & -bound) == bound) return (int)(((int64_t)bound * (int64_t)jr_next(r, 31)) >> 31);
    int bits, val;
    do {
        bits = jr_next(r, 31);
        val = bits % bound;
    } while ((int64_t)bits - val + (bound - 1) > INT32_MAX);
    return val;
}
static double jr_double(jrand *r) { return (double)(((int64_t)jr_next(r, 26) << 27) + jr_next(r, 27)) * 0x1.0p-53; }

/* fixed-order sum over block b of v[i] for the points of that block */
static double km_block_sum(const double *v, size_t n, size_t b) {
    double s[KM_T];
    for (int t = 0; t < KM_T; t++) {
        double a = 0.0;
        for (int j = 0; j < KM_PER; j++) {
            size_t i = b * KM_SPAN + (size_t)j * KM_T + t;
            if (i < n) a += v[i];
        }
        s[t] = a;
    }
    for (int st = KM_T / 2; st > 0; st >>= 1)
        for (int t = 0; t < st; t++) s[t] += s[t + st];
    return s[0];
}

static int km_taken(const size_t *taken, int nt, size_t i) {
    for (int q = 0; q < nt; q++)
        if (taken[q] == i) return 1;
    return 0;
}

/* One clustering of x[0..n): returns the number of centres; labels, centres,
 * counts and the WCSS out. */
static int km_run(const double *x, size_t n, int k, jrand *rng, int *lab, double *cen, double *cnt, double *wcss) {
    const size_t nb = (n + KM_SPAN - 1) / KM_SPAN;
    double *d2 = (double *)malloc(sizeof(double) * n), *tmp = (double *)malloc(sizeof(double) * n);
    double *part = (double *)malloc(sizeof(double) * nb);
    size_t taken[64];
    int nt = 0, have = 1;
    size_t first = (size_t)jr_int(rng, (int)n);
    cen[0] = x[first];
    taken[nt++] = first;
    while (have < k) {
        for (size_t i = 0; i < n; i++) {
            const double d = x[i] - cen[have - 1], e = d * d;
            d2[i] = have == 1 ? e : fmin(d2[i], e);
        }
        double sum = 0.0;
        for (size_t b = 0; b < nb; b++) { part[b] = km_block_sum(d2, n, b); sum += part[b]; }
        const double r = jr_double(rng) * sum;
        size_t pick = SIZE_MAX;
        double run = 0.0;
        for (size_t b = 0; b < nb && pick == SIZE_MAX; b++) {
            if (run + part[b] < r && b + 1 < nb) { run += part[b]; continue; }
            const size_t i0 = b * KM_SPAN, i1 = (i0 + KM_SPAN < n) ? i0 + KM_SPAN : n;
            for (size_t i = i0; i < i1; i++) {
                run += d2[i];
                if (run >= r && !km_taken(taken, nt, i)) { pick = i; break; }
            }
            if (pick == SIZE_MAX && run >= r)
                for (size_t i = i1; i-- > i0;)
                    if (!km_taken(taken, nt, i)) { pick = i; break; }
        }
        if (pick == SIZE_MAX)
            for (size_t i = n; i-- > 0;)
                if (!km_taken(taken, nt, i)) { pick = i; break; }
        if (pick == SIZE_MAX) break;
        cen[have++] = x[pick];
        taken[nt++] = pick;
    }
    k = have;
    double *sums = (double *)malloc(sizeof(double) * k), *next = (double *)malloc(sizeof(double) * k);
    for (size_t i = 0; i < n; i++) lab[i] = -1;
    /* assignment; returns changes, fills sums/cnt and the wcss in block order */
    #define KM_ASSIGN(changes_out)                                                                      \
        do {                                                                                            \
            long ch = 0;                                                                                \
            for (size_t i = 0; i < n; i++) {                                                            \
                int best = 0;                                                                           \
                double bd = (x[i] - cen[0]) * (x[i] - cen[0]);                                          \
                for (int c = 1; c < k; c++) {                                                           \
                    const double d = (x[i] - cen[c]) * (x[i] - cen[c]);                                 \
                    if (d < bd) { bd = d; best = c; }                                                   \
                }                                                                                       \
                if (lab[i] != best) ch++;                                                               \
                lab[i] = best;                                                                          \
                tmp[i] = bd;                                                                            \
            }                                                                                           \
            *wcss = 0.0;                                                                                \
            for (size_t b = 0; b < nb; b++) *wcss += km_block_sum(tmp, n, b);                           \
            for (int c = 0; c < k; c++) { sums[c] = 0.0; cnt[c] = 0.0; }                                \
            for (size_t b = 0; b < nb; b++)                                                             \
                for (int c = 0; c < k; c++) {                                                           \
                    for (size_t i = b * KM_SPAN; i < n && i < (b + 1) * KM_SPAN; i++)                   \
                        d2[i] = lab[i] == c ? x[i] : 0.0;                                               \
                    sums[c] += km_block_sum(d2, n, b);                                                  \
                    for (size_t i = b * KM_SPAN; i < n && i < (b + 1) * KM_SPAN; i++)                   \
                        d2[i] = lab[i] == c ? 1.0 : 0.0;                                                \
                    cnt[c] += km_block_sum(d2, n, b);                                                   \
                }                                                                                       \
            changes_out = ch;                                                                           \
        } while (0)
    long changes;
    KM_ASSIGN(changes);
    for (int it = 0; it < 1000; it++) {
        int empty = 0;
        for (int j = 0; j < k; j++) next[j] = cnt[j] > 0.0 ? sums[j] / cnt[j] : 0.0;
        for (int j = 0; j < k; j++) {
            if (cnt[j] > 0.0) continue;
            empty = 1;
            int sel = -1;
            double best = -HUGE_VAL;
            for (int q = 0; q < k; q++) {
                if (!(cnt[q] > 0.0)) continue;
                double s1 = 0.0, s2 = 0.0;
                for (size_t b = 0; b < nb; b++) {
                    for (size_t i = b * KM_SPAN; i < n && i < (b + 1) * KM_SPAN; i++)
                        tmp[i] = lab[i] == q ? fabs(x[i] - cen[q]) : 0.0;
                    s1 += km_block_sum(tmp, n, b);
                    for (size_t i = b * KM_SPAN; i < n && i < (b + 1) * KM_SPAN; i++)
                        tmp[i] = lab[i] == q ? fabs(x[i] - cen[q]) * fabs(x[i] - cen[q]) : 0.0;
                    s2 += km_block_sum(tmp, n, b);
                }
                const double var = cnt[q] > 1.0 ? (s2 - s1 * s1 / cnt[q]) / (cnt[q] - 1.0) : 0.0;
                if (var > best) { best = var; sel = q; }
            }
            const int want = jr_int(rng, (int)cnt[sel]);
            int seen = 0;
            for (size_t i = 0; i < n; i++)
                if (lab[i] == sel && seen++ == want) { next[j] = x[i]; cnt[sel] -= 1.0; break; }
        }
        for (int j = 0; j < k; j++) cen[j] = next[j];
        KM_ASSIGN(changes);
        if (changes == 0 && !empty) break;
    }
    #undef KM_ASSIGN
    free(d2); free(tmp); free(part); free(sums); free(next);
    return k;
}

/* ClassifyRedundancy_.run on a map: the interior (border cut) clustered into
 * k classes (or the elbow's k up to max_k), ranked by size (0 = largest, ties
 * in cluster order); the border is 0. Returns the number of classes. */
int orc_classify_redundancy(const float *map, int W, int H, int border, int k, int optimal_k, int max_k, int64_t seed,
                            float *out, double *wcss_out) {
    const int iw = W - 2 * border, ih = H - 2 * border;
    const size_t n = (size_t)iw * ih;
    double *x = (double *)malloc(sizeof(double) * n);
    int *lab = (int *)malloc(sizeof(int) * n);
    for (int y = 0; y < ih; y++)
        for (int xx = 0; xx < iw; xx++) x[(size_t)y * iw + xx] = (double)map[(y + border) * W + xx + border];
    jrand rng;
    jr_init(&rng, seed);
    double cen[64], cnt[64], wcss = 0.0;
    int kf = k;
    if (optimal_k) {
        double prev = DBL_MAX;
        kf = 1;
        for (int kt = 1; kt <= max_k; kt++) {
            km_run(x, n, kt, &rng, lab, cen, cnt, &wcss);
            if (wcss < prev) { prev = wcss; kf = kt; } else break;
        }
    }
    const int kc = km_run(x, n, kf, &rng, lab, cen, cnt, &wcss);
    int order[64], rank[64];
    for (int j = 0; j < kc; j++) order[j] = j;
    for (int a = 1; a < kc; a++) /* stable insertion sort, largest count first */
        for (int b = a; b > 0 && cnt[order[b]] > cnt[order[b - 1]]; b--) { int t = order[b]; order[b] = order[b - 1]; order[b - 1] = t; }
    for (int j = 0; j < kc; j++) rank[order[j]] = j;
    memset(out, 0, sizeof(float) * (size_t)W * H);
    for (int y = 0; y < ih; y++)
        for (int xx = 0; xx < iw; xx++) out[(y + border) * W + xx + border] = (float)rank[lab[(size_t)y * iw + xx]];
    *wcss_out = wcss;
    free(x);
    free(lab);
    return kc;
}

/* java.util.Random outputs for tests: next(bits) and nextDouble(). */
void orc_java_random_next(int64_t seed, int bits, int n, int32_t *out) {
    jrand r;
    jr_init(&r, seed);
    for (int i = 0; i < n; i++) out[i] = jr_next(&r, bits);
}
void orc_java_random_doubles(int64_t seed, int n, double *out) {
    jrand r;
    jr_init(&r, seed);
    for (int i = 0; i < n; i++) out[i] = jr_double(&r);
}

/* ------------------------------------------------------------------ */
/* Quadtree / octree variance stabilisation (java/QuadTree_.java,       */
/* java/OcTree_.java), literally: recursive build, FP32 sums in raster  */
/* order, Fisher test with the F quantile (same bisection of the        */
/* regularised incomplete beta as the library: Numerical Recipes'       */
/* continued fraction, modified Lentz), robust means, LTS variances by  */
/* sorting, SimpleRegression's updating sums, applyGATtree.             */
/* ------------------------------------------------------------------ */
static double orc_betacf(double a, double b, double x) {
    const double fpmin = 1e-300, eps = 1e-16;
    double qab = a + b, qap = a + 1.0, qam = a - 1.0, c = 1.0, d = 1.0 - qab * x / qap;
    if (fabs(d) < fpmin) d = fpmin;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m <= 1000000; m++) {
        int m2 = 2 * m;
        double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
        d = 1.0 + aa * d; if (fabs(d) < fpmin) d = fpmin;
        c = 1.0 + aa / c; if (fabs(c) < fpmin) c = fpmin;
        d = 1.0 / d; h *= d * c;
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
        d = 1.0 + aa * d; if (fabs(d) < fpmin) d = fpmin;
        c = 1.0 + aa / c; if (fabs(c) < fpmin) c = fpmin;
        d = 1.0 / d;
        double del = d * c;
        h *= del;
        if (fabs(del - 1.0) < eps) break;
    }
    return h;
}
static double orc_ibeta(double a, double b, double x) {
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    double front = exp(lgamma(a + b) - lgamma(a) - lgamma(b) + a * log(x) + b * log1p(-x));
    if (x < (a + 1.0) / (a + b + 2.0)) return front * orc_betacf(a, b, x) / a;
    return 1.0 - front * orc_betacf(b, a, 1.0 - x) / b;
}
double orc_f_quantile(double p, double df) {
    double a = 0.5 * df, lo = 0.0, hi = 1.0;
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (orc_ibeta(a, a, mid) < p) lo = mid; else hi = mid;
    }
    double x = 0.5 * (lo + hi);
    return x / (1.0 - x);
}

typedef struct { int x, y, z, w, h, d; } tbox;
typedef struct {
    const float *img;
    int W, H, D, oct, min_size, max_iter;
    float alpha, frac;
    tbox *leaves;
    int n_leaves, cap;
} tctx;

static float tree_block_var(const tctx *t, tbox b) {
    /* 2D: Utils.getMeanAndVarBlock2D (FP32); 3D: getMeanAndVarBlock3D (FP64) */
    const long n = (long)b.w * b.h * b.d;
    if (!t->oct) {
        float mean = 0.0f, sq = 0.0f;
        for (int y = b.y; y < b.y + b.h; y++)
            for (int x = b.x; x < b.x + b.w; x++) {
                float v = t->img[(long)y * t->W + x];
                mean += v;
                sq += v * v;
            }
        mean = mean / (float)n;
        return sq / (float)n - mean * mean;
    }
    double mean = 0.0, sq = 0.0;
    for (int z = b.z; z < b.z + b.d; z++)
        for (int y = b.y; y < b.y + b.h; y++)
            for (int x = b.x; x < b.x + b.w; x++) {
                double v = (double)t->img[((long)z * t->H + y) * t->W + x];
                mean += v;
                sq += v * v;
            }
    mean = mean / n;
    return (float)(sq / n - mean * mean);
}

static float tree_noise_var(const tctx *t, tbox b) {
    const int W = t->W, H = t->H, D = t->D;
    const float l = t->oct ? 7.0f : 5.0f;
    const float scale = (float)(1.0 / sqrt((double)(l * l + l)));
    const long n = (long)b.w * b.h * b.d;
    float *r = (float *)malloc(sizeof(float) * (size_t)n);
    long k = 0;
    for (int z = b.z; z < b.z + b.d; z++)
        for (int y = b.y; y < b.y + b.h; y++)
            for (int x = b.x; x < b.x + b.w; x++) {
                const long p = ((long)z * H + y) * W + x;
                float lap = l * t->img[p];
                if (x > 0) lap -= t->img[p - 1];
                if (x < W - 1) lap -= t->img[p + 1];
                if (y > 0) lap -= t->img[p - W];
                if (y < H - 1) lap -= t->img[p + W];
                if (t->oct) {
                    if (z > 0) lap -= t->img[p - (long)W * H];
                    if (z < D - 1) lap -= t->img[p + (long)W * H];
                }
                r[k++] = lap * scale;
            }
    float s = 0.0f;
    for (long i = 0; i < n; i++) s += r[i];
    const float m = s / (float)n;
    float ss = 0.0f;
    for (long i = 0; i < n; i++) ss += (float)pow((double)r[i] - (double)m, 2.0);
    free(r);
    return ss / ((float)n - 1.0f);
}

static void tree_build(tctx *t, tbox b) {
    const float vz = tree_block_var(t, b), ve = tree_noise_var(t, b);
    const float ratio = fminf(vz, ve) / fmaxf(vz, ve);
    const long df = (long)b.w * b.h - 1;
    const float thr = df >= 1 ? (float)orc_f_quantile((double)t->alpha, (double)df) : 0.0f;
    const int divide = ratio < thr;
    if (b.w <= t->min_size || b.h <= t->min_size || (t->oct && b.d <= t->min_size) || !divide) {
        if (t->n_leaves == t->cap) {
            t->cap = t->cap ? 2 * t->cap : 64;
            t->leaves = (tbox *)realloc(t->leaves, sizeof(tbox) * t->cap);
        }
        t->leaves[t->n_leaves++] = b;
        return;
    }
    const int hw = b.w / 2, hh = b.h / 2, hd = t->oct ? b.d / 2 : 1;
    const int nch = t->oct ? 8 : 4;
    for (int k = 0; k < nch; k++) {
        tbox c = {b.x + ((k & 1) ? hw : 0), b.y + ((k & 2) ? hh : 0), b.z + ((k & 4) ? hd : 0), hw, hh, hd};
        tree_build(t, c);
    }
}

static float tree_robust_mean(const tctx *t, tbox b) {
    float mean = 0.0f, var = 0.0f;
    long n = 0;
    for (int z = b.z; z < b.z + b.d; z++)
        for (int y = b.y; y < b.y + b.h; y++)
            for (int x = b.x; x < b.x + b.w; x++) {
                float v = t->img[((long)z * t->H + y) * t->W + x];
                mean += v;
                var += (v - mean) * (v - mean);
                n++;
            }
    mean /= (float)n;
    var /= (float)(n - 1);
    var = fmaxf(var, ORC_EPS);
    float prev;
    int it = 0;
    do {
        prev = mean;
        float ws = 0.0f, wv = 0.0f;
        for (int z = b.z; z < b.z + b.d; z++)
            for (int y = b.y; y < b.y + b.h; y++)
                for (int x = b.x; x < b.x + b.w; x++) {
                    float v = t->img[((long)z * t->H + y) * t->W + x];
                    float w = (float)exp(-((double)(v - mean) * (double)(v - mean)) / (2.0 * (double)var));
                    ws += w;
                    wv += w * v;
                }
        mean = wv / fmaxf(ws, ORC_EPS);
        it++;
    } while (fabsf(mean - prev) > 1e-5f && it < t->max_iter);
    return mean;
}

static int cmp_f(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

static float tree_lts(const tctx *t, tbox b, float m) {
    const long n = (long)b.w * b.h * b.d;
    float *r = (float *)malloc(sizeof(float) * (size_t)n);
    long k = 0;
    for (int z = b.z; z < b.z + b.d; z++)
        for (int y = b.y; y < b.y + b.h; y++)
            for (int x = b.x; x < b.x + b.w; x++) {
                float v = t->img[((long)z * t->H + y) * t->W + x];
                r[k++] = (v - m) * (v - m);
            }
    qsort(r, (size_t)n, sizeof(float), cmp_f);
    const int h = (int)floorf(t->frac * (float)n);
    float s = 0.0f;
    for (int i = 0; i < h; i++) s += r[i];
    free(r);
    return s / ((float)h + ORC_EPS);
}

/* Returns the number of leaves (or -1 if the regression has no slope);
 * leaves (x, y, z, w, h, d each), means and variances go to the out arrays
 * when given (capacity max_leaves). img is transformed in place. */
int orc_gat_tree(float *img, int W, int H, int D, int oct, int min_size, float alpha, int max_iter, float frac,
                 double *g0_out, double *edc_out, int *boxes_out, float *means_out, float *vars_out, int max_leaves) {
    tctx t = {img, W, H, D, oct, min_size, max_iter, alpha, frac, NULL, 0, 0};
    tbox root = {0, 0, 0, W, H, D};
    tree_build(&t, root);
    double sx = 0, sy = 0, sxx = 0, sxy = 0, xbar = 0, ybar = 0;
    for (int i = 0; i < t.n_leaves; i++) {
        const float m = tree_robust_mean(&t, t.leaves[i]);
        const float v = tree_lts(&t, t.leaves[i], m);
        if (i < max_leaves) {
            if (boxes_out) memcpy(boxes_out + 6 * i, &t.leaves[i], sizeof(tbox));
            if (means_out) means_out[i] = m;
            if (vars_out) vars_out[i] = v;
        }
        const double x = m, y = v;
        if (i == 0) { xbar = x; ybar = y; }
        else {
            const double nn = (double)i, f1 = 1.0 + nn, f2 = nn / (1.0 + nn), dx = x - xbar, dy = y - ybar;
            sxx += dx * dx * f2; sxy += dx * dy * f2; xbar += dx / f1; ybar += dy / f1;
        }
        sx += x; sy += y;
    }
    const int nl = t.n_leaves;
    free(t.leaves);
    if (nl < 2 || fabs(sxx) < 10 * DBL_MIN) return -1;
    const double g0 = sxy / sxx, edc = (sy - g0 * sx) / nl, c = 0.375 * g0 * g0 + edc;
    for (long i = 0; i < (long)W * H * D; i++) {
        double v = (double)img[i];
        v = (g0 * v + c) < 0.0 ? 0.0 : (2.0 / g0) * sqrt(g0 * v + c);
        img[i] = (float)v;
    }
    *g0_out = g0;
    *edc_out = edc;
    return nl;
}

/* ------------------------------------------------------------------ */
/* Block-map Hu distance (this library's north-star Hu metric; the     */
/* reference outputs only Hu1, cl/kernelGetPatchHu2D.cl:267): the L2    */
/* distance between the seven Hu invariants (Hu 1962) of each block and */
/* of the reference block, FP64. Intensities are min-max normalised     */
/* over the ellipse (all invariants 0 for a flat block); eta_pq =       */
/* mu_pq / m00^(1 + (p + q) / 2) from the central moments about the     */
/* intensity centroid, the offsets taken relative to the block centre.  */
/* ------------------------------------------------------------------ */
static void orc_hu7_vec(const double *x, const int *dx, const int *dy, int K, double *h) {
    double mn = x[0], mx = x[0];
    for (int k = 1; k < K; k++) {
        if (x[k] < mn) mn = x[k];
        if (x[k] > mx) mx = x[k];
    }
    for (int i = 0; i < 7; i++) h[i] = 0.0;
    double span = mx - mn;
    if (!(span > 0.0)) return;
    double m00 = 0.0, m10 = 0.0, m01 = 0.0;
    for (int k = 0; k < K; k++) {
        double v = (x[k] - mn) / span;
        m00 += v;
        m10 += (double)dx[k] * v;
        m01 += (double)dy[k] * v;
    }
    double cx = m10 / m00, cy = m01 / m00;
    double u20 = 0, u11 = 0, u02 = 0, u30 = 0, u21 = 0, u12 = 0, u03 = 0;
    for (int k = 0; k < K; k++) {
        double v = (x[k] - mn) / span;
        double a = (double)dx[k] - cx, b = (double)dy[k] - cy;
        double a2 = a * a, b2 = b * b;
        u20 += a2 * v;
        u11 += (a * b) * v;
        u02 += b2 * v;
        u30 += (a2 * a) * v;
        u21 += (a2 * b) * v;
        u12 += (a * b2) * v;
        u03 += (b2 * b) * v;
    }
    double s2 = m00 * m00, s3 = s2 * sqrt(m00);
    double n20 = u20 / s2, n11 = u11 / s2, n02 = u02 / s2;
    double n30 = u30 / s3, n21 = u21 / s3, n12 = u12 / s3, n03 = u03 / s3;
    double p = n30 + n12, q = n21 + n03, r = n30 - 3.0 * n12, s = 3.0 * n21 - n03, d = n20 - n02;
    h[0] = n20 + n02;
    h[1] = d * d + 4.0 * (n11 * n11);
    h[2] = r * r + s * s;
    h[3] = p * p + q * q;
    h[4] = r * p * (p * p - 3.0 * (q * q)) + s * q * (3.0 * (p * p) - q * q);
    h[5] = d * (p * p - q * q) + 4.0 * n11 * p * q;
    h[6] = s * p * (p * p - 3.0 * (q * q)) - r * q * (3.0 * (p * p) - q * q);
}

/* Raw map (interior pixels; border 0) and the reference 7-vector. */
void orc_block_hu7(const float *img, int W, int H, int bw, int bh, const float *ref_pixels, double *ref_h,
                   double *out) {
    int rw = bw / 2, rh = bh / 2;
    int *dx = (int *)malloc(sizeof(int) * bw * bh), *dy = (int *)malloc(sizeof(int) * bw * bh);
    int K = 0;
    for (int y = -rh; y <= rh; y++)
        for (int x = -rw; x <= rw; x++)
            if (in_ellipse(x, y, rw, rh)) { dx[K] = x; dy[K] = y; K++; }
    double *rv = (double *)malloc(sizeof(double) * K);
    for (int k = 0; k < K; k++) rv[k] = (double)ref_pixels[k];
    orc_hu7_vec(rv, dx, dy, K, ref_h);
    #pragma omp parallel for schedule(static)
    for (int gy = 0; gy < H; gy++) {
        double v[1024], h[7];
        for (int gx = 0; gx < W; gx++) {
            out[gy * W + gx] = 0.0;
            if (gx < rw || gx >= W - rw || gy < rh || gy >= H - rh) continue;
            for (int k = 0; k < K; k++) v[k] = (double)img[(gy + dy[k]) * W + gx + dx[k]];
            orc_hu7_vec(v, dx, dy, K, h);
            double s2 = 0.0;
            for (int i = 0; i < 7; i++) { double t = h[i] - ref_h[i]; s2 += t * t; }
            out[gy * W + gx] = sqrt(s2);
        }
    }
    free(rv);
    free(dx);
    free(dy);
}
