/*
 * libsred: B200 (sm_100a) implementation of SReD's block-correlation path.
 *
 * C ABI only: plain pointers and sizes, no C++ or torch types. Every entry
 * point returns an sred_status and never aborts the process. Host pointers
 * ("const float* img", "float* out") are caller-owned host memory; functions
 * with the _device suffix take device pointers on the given CUDA stream.
 *
 * Reference interfaces replaced (paths relative to the SReD repository root):
 *   java/  = src/main/java/
 * Metric arguments are the reference's dialog strings, matched exactly.
 */
#ifndef SRED_H
#define SRED_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SRED_OK = 0,
    SRED_ERR_ARG = 1,            /* bad size/argument; the reference throws or IJ.error()s */
    SRED_ERR_UNKNOWN_METRIC = 2, /* the reference returns null (java/CLUtils.java:2193-2195) */
    SRED_ERR_NODEV = 3,
    SRED_ERR_OOM = 4,
    SRED_ERR_LAUNCH = 5,
    SRED_ERR_TIMEOUT = 6,
    SRED_ERR_INTERNAL = 7,
    SRED_ERR_INVALID_INPUT = 8   /* NaN/Inf pixel in a noise tile (java/Utils.java:886-889) */
} sred_status;

/* Contraction engine of the global map. SRED_ENGINE_TC: split-BF16 tcgen05
 * tensor-core Gram with FP32 accumulation (u = hi + mid, or hi + mid + lo
 * when 6K <= 128 and for NRMSE); SRED_ENGINE_FP32: plain FP32 CUDA-core Gram.
 * Both share moments, the symmetric schedule (each unordered block pair
 * evaluated once) and the fused epilogue. Abs-diff needs no contraction and
 * runs on the FP32 engine's kernel; a map whose operands do not fit the
 * tensor-core kernel's shared memory (K' above 576) falls back to the FP32
 * engine, where NRMSE accumulates |u_p - u_q|^2 directly. */
typedef enum { SRED_ENGINE_TC = 0, SRED_ENGINE_FP32 = 1 } sred_engine;

typedef struct sred_ctx sred_ctx;

/* Timing and counts of the last global-map call. */
typedef struct {
    int64_t n_blocks;          /* interior blocks (W-2rw)*(H-2rh) */
    int64_t n_relevant;        /* blocks with sigma^2 >= threshold (enter the sums) */
    int64_t n_flat;            /* relevant blocks with sigma == 0 */
    double pairs;              /* n_relevant^2: block pairs the map is defined over */
    float noise_var;           /* FILTER_PARAM (java/Utils.java:790-837) */
    float threshold;           /* noise_var * relevance constant */
    float n_pixels;            /* java/GlobalRepetition2D_.java:133-140 */
    int k;                     /* ellipse block size */
    int engine;                /* sred_engine used */
    double ms_moments, ms_gram, ms_finalize, ms_total; /* CUDA-event times */
    int launches;              /* kernels this call launched */
} sred_run_info;

/* Context: owns the device, a stream and reusable workspaces.
 * One context per host thread; calls on one context are serialised. */
sred_status sred_create(int device_ordinal, sred_ctx **out);
sred_status sred_destroy(sred_ctx *ctx);
sred_status sred_set_engine(sred_ctx *ctx, int engine);
/* Messages of the context (errors, and one line per global map with its
 * size, relevant blocks, engine and time) are passed to cb on the calling
 * thread; NULL turns logging off. The reference reports through IJ.log /
 * IJ.error (java/GlobalRepetition2D_.java, java/CLUtils.java); a host binds
 * this callback to its own log. */
sred_status sred_set_log_callback(sred_ctx *ctx, void (*cb)(const char *message, void *user), void *user);
const char *sred_status_string(sred_status s);
const char *sred_last_error(sred_ctx *ctx);

/* Ellipse block size K for a bw x bh block (java/GlobalRepetition2D_.java:102-111). */
int sred_block_size(int bw, int bh);

/* Replaces CLUtils.getLocalStatistics2D (java/CLUtils.java:376-467) and
 * cl/kernelGetLocalStatistics2D.cl: per-pixel ellipse-block mean and (K-1)
 * standard deviation in FP32, reference evaluation order; border pixels 0. */
sred_status sred_local_statistics_2d(sred_ctx *ctx, const float *img, int w, int h, int bw, int bh,
                                     float *local_means, float *local_stds);

/* Replaces Utils.getMeanNoiseVar2D (java/Utils.java:790-837). */
sred_status sred_mean_noise_var_2d(sred_ctx *ctx, const float *img, int w, int h, float *noise_var);

/* Replaces Utils.getRelevanceMask (java/Utils.java:944-968): mask[w*h] in {0,1},
 * threshold = noise_var * relevance_constant. */
sred_status sred_relevance_mask_2d(sred_ctx *ctx, const float *img, int w, int h, int bw, int bh,
                                   const float *local_stds, float relevance_constant, float *mask,
                                   float *threshold, float *noise_var);

/* Replaces CLUtils.calculateGlobalRepetitionMap2D (java/CLUtils.java:2174-2196)
 * and the four getGlobal*2D methods it dispatches to (:1680-2156), with the
 * same inputs: the preprocessed image, block size, the FP32 local statistics
 * of CLLocalStatistics (relevance and flat-block decisions are taken on
 * local_stds, as the reference kernels take them), the RelevanceMask fields
 * (mask, relevance constant, threshold, noise variance) and nPixels.
 * metric: "Pearson's R", "SSIM", "NRMSE" or "Abs. diff. of StdDevs".
 * out receives the finished map (w*h), including the host post-processing. */
sred_status sred_calculate_global_repetition_map_2d(
    sred_ctx *ctx, const char *metric, const float *img, int w, int h, int bw, int bh, int block_size,
    const float *local_means, const float *local_stds, const float *mask, float relevance_constant,
    float threshold, float noise_var, float n_pixels, int normalize_output, float *out,
    sred_run_info *info);

/* The whole command after preprocessing, as GlobalRepetition2D_.run does it
 * (java/GlobalRepetition2D_.java:97-145): K, local statistics, relevance
 * mask, nPixels and the map, all on the device.
 *
 * Run-to-run determinism of every global map: each block's pair sums are
 * FP32 partial sums (per tile row or column) added into FP64 totals with
 * atomic adds, in an order that varies between runs. The FP64 totals can
 * differ in their last bits (relative 1e-16, against the 2^-24 rounding of
 * the FP32 map), so a map repeats bit for bit except where a total lies
 * within that distance of an FP32 rounding boundary. */
sred_status sred_global_map_2d(sred_ctx *ctx, const char *metric, const float *img, int w, int h,
                               int bw, int bh, float relevance_constant, int normalize_output,
                               float *out, sred_run_info *info);

/* Sharded global map (no counterpart in the reference): the map of
 * sred_global_map_2d_device split across n_shards processes, usually one
 * per GPU. The all-pairs contraction evaluates each unordered pair of
 * relevant blocks once, as tiles of the upper triangle of the pair matrix
 * grouped into work items (a tile adds its pair terms to both blocks' sums);
 * shard s of S takes work items [I s / S, I (s + 1) / S) of the I items of
 * the engine's default launch shape. Phase 1, on every shard: the moment
 * pass, relevance mask and compaction (all of them, on every shard), then
 * the pair terms of this shard's tiles, added into d_sums (device memory,
 * capacity in doubles >= 2 x relevant blocks; the interior pixel count
 * always suffices) laid out as [num | den] over the relevant non-flat
 * blocks; info->n_relevant - info->n_flat is their count. Every shard's
 * sums cover part of every block's pairs. The caller then sums d_sums over
 * the shards (one all-reduce, e.g. NCCL) and calls phase 2 on every shard
 * that needs the map, with the summed buffer: finalisation and normalisation
 * into d_out. No other call may use the context between the two phases
 * (phase 2 then fails with SRED_ERR_ARG). */
sred_status sred_global_map_2d_shard_sums(sred_ctx *ctx, const char *metric, const float *d_img, int w, int h,
                                          int bw, int bh, float relevance_constant, int shard, int n_shards,
                                          double *d_sums, size_t capacity, void *stream, sred_run_info *info);
sred_status sred_global_map_2d_shard_finish(sred_ctx *ctx, const double *d_sums, int normalize_output,
                                            float *d_out, void *stream, sred_run_info *info);

/* One map of a batch (sred_global_map_2d_batch): the arguments of
 * sred_global_map_2d, and the job's own status on return. */
typedef struct {
    const char *metric;
    const float *img;          /* host, w*h */
    int w, h, bw, bh;
    float relevance_constant;
    int normalize_output;
    float *out;                /* host, w*h */
    sred_run_info *info;       /* nullable */
    int status;                /* written: sred_status of this job */
} sred_job;

/* Many global maps in one call (no counterpart in the reference, whose
 * command computes one map per invocation): jobs run on `n_workers` (1..8)
 * host threads, each with its own CUDA stream and workspaces, so that one
 * map's host steps and transfers overlap another map's kernels. Each map is
 * what sred_global_map_2d returns for it (up to the FP64 sum order described
 * there). Returns SRED_OK if
 * every job succeeded, else the first failing job's status. */
sred_status sred_global_map_2d_batch(sred_ctx *ctx, sred_job *jobs, int n_jobs, int n_workers);

/* Same as sred_global_map_2d with device-resident input and output on
 * `stream` (a cudaStream_t; NULL = the context's stream). The call returns
 * when the map is complete. */
sred_status sred_global_map_2d_device(sred_ctx *ctx, const char *metric, const float *d_img, int w,
                                      int h, int bw, int bh, float relevance_constant,
                                      int normalize_output, float *d_out, void *stream,
                                      sred_run_info *info);

/* Replaces CLUtils.calculateBlockRepetitionMap2D (java/CLUtils.java:995-1010)
 * and getBlock{Pearson,Ssim,Nrmse,AbsDiffStds}2D (:486-981). ref_pixels,
 * block_size, bw, bh, ref_mean and ref_std are the ReferenceBlock2D fields
 * (java/Utils.java:108-216), passed through unchanged. metric:
 * "Pearson's R", "SSIM", "NRMSE (inverted)", "Abs. Diff. of StdDevs." (the
 * reference's four), or one of four without a dialog entry in the
 * reference, all post-processed like Pearson:
 *   "Cosine"            raw-vector cosine similarity;
 *   "Hu moments"        cl/kernelGetPatchHu2D.cl (sqrt(hu1_ref * hu1_block))
 *                       with the reference block's ellipse pixels normalised
 *                       the way that kernel normalises each block
 *                       (mean-subtract, min-max to [0, 1], FP64);
 *   "Phase correlation" the peak distance of the normalised cross-power
 *                       spectrum of cl/kernelGetPhaseCorrelationMap.cl
 *                       (repaired as for sred_phase_correlation_map_2d)
 *                       between the reference block / (ref_std + eps) and
 *                       each block, normalised with its FP32 local mean and
 *                       std, both restricted to the ellipse, through the
 *                       exact DFT of the block (twiddle angles 2 pi jk / n
 *                       reduced modulo n, where the kernel takes pi as a
 *                       float and does not reduce); bw, bh <= 15;
 *   "Hu distance"       the L2 distance between the seven Hu moment
 *                       invariants (Hu 1962) of each block's ellipse pixels
 *                       and those of the reference block, both min-max
 *                       normalised to [0, 1] first, FP64 (the reference's
 *                       Hu kernels output the first invariant only). */
sred_status sred_calculate_block_repetition_map_2d(sred_ctx *ctx, const char *metric, const float *img,
                                                   int w, int h, const float *ref_pixels, int block_size,
                                                   int bw, int bh, float ref_mean, float ref_std,
                                                   float relevance_constant, int normalize_output,
                                                   float *out);

/* Device-resident variant over a stack of `frames` images (the time-lapse
 * loop of java/BlockRepetition2D_.java:95-130): d_img is frames*w*h, d_out the
 * same. */
sred_status sred_block_map_2d_device(sred_ctx *ctx, const char *metric, const float *d_img, int w,
                                     int h, int frames, const float *ref_pixels, int block_size, int bw,
                                     int bh, float ref_mean, float ref_std, float relevance_constant,
                                     int normalize_output, float *d_out, void *stream);

/* Host-buffer variant over a stack of `frames` images (the same time-lapse
 * loop): img and out are frames*w*h floats in host memory, each frame mapped
 * and normalised on its own, exactly as sred_block_map_2d_device maps them.
 * The stack moves in chunks of chunk_frames frames (0: about 32 MiB per
 * chunk) through two device slots, so the upload of one chunk, the map of the
 * previous one and the download of the one before run at the same time; with
 * page-locked host buffers the copies run concurrently with the kernels.
 * Returns when out is complete (or, on an error, when no copy touches img or
 * out any more). */
sred_status sred_block_map_2d_stack(sred_ctx *ctx, const char *metric, const float *img, int w, int h,
                                    int frames, const float *ref_pixels, int block_size, int bw, int bh,
                                    float ref_mean, float ref_std, float relevance_constant,
                                    int normalize_output, int chunk_frames, float *out);

/* Replaces Utils.getReferenceBlock2D (java/Utils.java:557-639) for a block
 * image already converted to float: ellipse-flatten, min-max, mean-subtract,
 * std. pixels must hold sred_block_size(bw, bh) floats. */
sred_status sred_reference_block_2d(const float *block_img, int bw, int bh, float *pixels,
                                    int *block_size, float *mean, float *std);

/* Variance stabilisation of the input image (the default "stabiliseNoiseVariance"
 * step of java/Utils.java:674-684, Simplex method).
 *
 * Replaces VarianceStabilisingTransform2D_.getGAT
 * (java/VarianceStabilisingTransform2D_.java:136-151), in place on host memory:
 * v = (2 / gain) sqrt(gain v + c), c = 3/8 gain^2 + sigma^2 - gain offset, 0
 * where gain v + c < 0; double arithmetic, float result. */
sred_status sred_gat_2d(sred_ctx *ctx, float *img, int w, int h, double gain, double sigma, double offset);

/* The objective of GATMinimizer2D.userFunction (java/GATMinimizer2D.java): the
 * image transformed as its applyGAT does, cut into width/6 x height/6-pixel
 * blocks, sum over blocks of (block variance - 1)^2 / blocks. w, h >= 12. */
sred_status sred_gat_objective_2d(sred_ctx *ctx, const float *img, int w, int h, double gain, double sigma,
                                  double offset, double *error);

/* Replaces GATMinimizer2D.run: minimises that objective over (gain, sigma,
 * offset) from the values passed in (the reference starts at 1, 10, 100 with
 * steps 1, 10, 100 and 5000 iterations), with a Nelder-Mead simplex of this
 * library (the reference uses ImageJ's Minimizer, which is not part of SReD,
 * so the fitted values agree with the reference's only as minimisers of the
 * same objective). On return the three values are the fit; error (nullable)
 * receives its objective. */
sred_status sred_gat_fit_2d(sred_ctx *ctx, const float *img, int w, int h, int max_iter, double *gain,
                            double *sigma, double *offset, double *error);

/* 3D variance stabilisation (java/GATMinimizer3D.java). sred_gat_3d:
 * getGAT over all w*h*d voxels, in place. sred_gat_objective_3d:
 * GATMinimizer3D.userFunction: NaN unless gain > 0, sigma >= 0, offset >= 0;
 * blocks of width/6 x height/6 x depth/6 voxels (halved along an axis with
 * fewer than 2 blocks), per-block variance of the transformed voxels (FP64
 * sums), sum over blocks of (variance - 1)^2 / blocks. sred_gat_fit_3d: the
 * simplex of sred_gat_fit_2d over that objective (an objective of NaN ranks
 * last); the reference's command starts it at gain 0, sigma 100, offset 0
 * (java/Utils.java:1222). */
sred_status sred_gat_3d(sred_ctx *ctx, float *vol, int w, int h, int d, double gain, double sigma, double offset);
sred_status sred_gat_objective_3d(sred_ctx *ctx, const float *vol, int w, int h, int d, double gain, double sigma,
                                  double offset, double *error);
sred_status sred_gat_fit_3d(sred_ctx *ctx, const float *vol, int w, int h, int d, int max_iter, double *gain,
                            double *sigma, double *offset, double *error);

/* Replaces Utils.normalizeImage2D (java/Utils.java:985-1031) on host memory.
 * mask may be NULL. SRED_ERR_ARG for a non-binary mask. */
sred_status sred_normalize_image_2d(float *img, int w, int h, int border_w, int border_h,
                                    const float *mask);

/* The reference's shape-metric kernels, which it ships in
 * src/main/resources/ but never loads from its Java code. Host memory in and
 * out; border pixels of `out` are 0.
 *
 * Replaces cl/kernelGetPatchHu2D.cl:11-282: for every interior pixel
 * (float)sqrt(hu1(patch) * hu1(block)), FP64, with the kernel's own
 * arithmetic (raw moments at 1-based and central moments at 0-based
 * coordinates; the block mean summed over the square minus its four corners
 * and divided by patch_size; min-max remap over the ellipse). patch: the
 * bw x bh grid the kernel reads at the ellipse positions; patch_size: its
 * $PATCH_SIZE$ (the reference's Java convention is the ellipse count K). */
sred_status sred_patch_hu_map_2d(sred_ctx *ctx, const float *patch, const float *img, int w, int h, int bw,
                                 int bh, int patch_size, float *out);

/* Replaces cl/kernelGetHuMap.cl:15-172 (speedUp off): for every interior
 * pixel p, the sum over every interior pixel q of |hu_q - hu_p| *
 * (100^s - 1) / 99 with s = 1 - |std_p - std_q| / (|std_p| + |std_q| + eps),
 * where hu is the FP32 invariant(2,0) + invariant(0,2) of the whole square
 * block minus the local mean. FP32 terms, FP64 sums. local_means/local_stds
 * are CLLocalStatistics' buffers (sred_local_statistics_2d). */
sred_status sred_hu_map_2d(sred_ctx *ctx, const float *img, const float *local_means, const float *local_stds,
                           int w, int h, int bw, int bh, float *out);

/* Replaces cl/kernelGetPhaseCorrelationMap.cl:13-179 (speedUp off), which does
 * not compile as shipped, with its three defects repaired: no unique-pixel
 * pre-filter (nUnique is never defined, :27), real-valued DFT phases (the
 * shipped (1*i*ii/bW) divides integers, :66/:101/:138) and the peak search
 * indexed by the block width (:150 uses the image width). For every interior
 * pixel p, the sum over every interior q of |peak_pq| * weight(std_p, std_q),
 * peak_pq the 1-based position of the first maximum above 0 of the inverse
 * DFT of the normalised cross-power spectrum of the two whole square blocks,
 * each normalised as (x - mean) / (std + eps). FP64, FP64 sums. bw, bh <= 15;
 * the cost grows as (interior pixels)^2 * bw * bh * (bw + bh). */
sred_status sred_phase_correlation_map_2d(sred_ctx *ctx, const float *img, const float *local_means,
                                          const float *local_stds, int w, int h, int bw, int bh, float *out);

/* Block map that allocates nothing (no counterpart in the reference): for
 * callers that cannot call cudaMalloc, such as hosts whose runtime owns the
 * device allocator, or loops that must not touch the allocator once started.
 * Same result as sred_block_map_2d_device with relevance_constant 0; needs no
 * context. Runs on the current device and on `stream` (NULL = the default
 * stream) and synchronises that stream before it returns, so the map is
 * complete then. Scratch is a fixed device array of about 4 MiB that every
 * GPU loading this library holds until exit; the limits are frames <= 4096,
 * for NRMSE frames * w * h <= 1,048,576, and a block whose image tile with
 * halo fits in 48 KB of shared memory (every block up to 25 x 25; a 3 x 401
 * block does not) (SRED_ERR_ARG beyond them). The first call on a device
 * looks the array's device address up (make that first call before any
 * stream capture). Every call shares the array, so calls that overlap on the
 * GPU race. */
sred_status sred_block_map_2d_device_noalloc(const char *metric, const float *d_img, int w, int h,
                                             int frames, const float *ref_pixels, int block_size, int bw,
                                             int bh, float ref_mean, float ref_std, int normalize_output,
                                             float *d_out, void *stream);

/* Diagnostics of the contraction engines (no counterpart in the reference):
 * for caller-given vectors u (n x k, row-major) and weights w1, w2,
 * num[p] = sum_q <u_p, u_q> w1[p] w1[q] and den[p] = sum_q (w2[p] + w2[q]),
 * symmetric pair terms like the maps' own, computed by the
 * chosen engine's all-pairs kernel (the tensor-core engine splits u into
 * bf16 hi/lo without normalising it). */
sred_status sred_debug_gram_rowdot(sred_ctx *ctx, int engine, const float *u, const float *w1,
                                   const float *w2, int n, int k, double *num, double *den);

/* Test hook of the tensor-core engine's bounded waits (no counterpart in the
 * reference; the reference's host raises a RuntimeException when its OpenCL
 * set-up fails, java/CLUtils.java:175-180): every pipeline wait of later
 * global maps on this context gives up after timeout_ns (0: the default 4 s),
 * and withhold_tile >= 0 makes the copy producer stop before that tile's
 * operands, so the waits run out with no copy in flight and the call returns
 * SRED_ERR_TIMEOUT with the context still usable. withhold_tile = -1 restores
 * normal operation. */
sred_status sred_debug_set_tc_wait(sred_ctx *ctx, unsigned long long timeout_ns, long long withhold_tile);

/* Launch-shape tuner of the tensor-core engine (no counterpart in the
 * reference, whose OpenCL kernels run one fixed work-group size,
 * java/CLUtils.java:432-433). A global map's contraction can run as
 * 128 x 256 or 128 x 128 tiles, with each tile's A operand resident or
 * streamed through a ring of 16 KB chunks, and with 32, 16, 8 or 4 row blocks
 * per run of work items. The process keeps one table, shared by every context:
 * key (K' = padded contraction length, metric code, size class of the
 * contracted block count n: 0 below 65,536, 1 below 262,144, else 2) ->
 * shape. A map whose key is in the table runs that shape; other maps run the
 * default shape (128 x 256, A resident when it fits, 32 row blocks).
 *
 * sred_set_gram_tuning(ctx, 1) makes later unsharded maps on ctx (and its
 * batch workers) whose key is missing time every shape on their own
 * operands, each from zeroed sums, store the fastest, then compute the map
 * with it: the map equals the one the stored shape gives. Maps running at
 * the same time on other streams perturb the timings; tune on one context at
 * a time. Sharded maps always run the default shape. */
sred_status sred_set_gram_tuning(sred_ctx *ctx, int on);

/* Copies at most `cap` table entries: entries[6 i .. 6 i + 5] = K', metric
 * code, size class, tile columns (256 or 128), A resident (1) or chunk ring
 * (0), row blocks per run; ms[i] = that shape's timed contraction in ms.
 * Returns the number of entries in the table (call with cap 0 to size). */
int sred_gram_tuning_entries(int *entries, float *ms, int cap);

/* Stores one entry (a shape read back from a saved table); SRED_ERR_ARG when
 * the shape does not fit K' or the size class is not 0, 1 or 2. */
sred_status sred_gram_tuning_set(int kq, int metric, int size_class, int bn, int tr, int max_l, float ms);

/* Empties the table. */
sred_status sred_gram_tuning_clear(void);

/* ---------------------------------------------------------------------
 * 3D block repetition maps. Volumes are w x h x d floats, x fastest then y
 * then z (the reference's flattened ImageStack, index w*h*z + y*w + x); the
 * block is the ellipsoid inscribed in an odd bw x bh x bd box (each >= 3).
 * --------------------------------------------------------------------- */

/* Ellipsoid block size K (java/Utils.java:1075-1085, float arithmetic). */
int sred_block_size_3d(int bw, int bh, int bd);

/* Replaces Utils.getReferenceBlock3D (java/Utils.java:1047-1160) for a block
 * already converted to float (bd slices of bh x bw): ellipsoid-flatten,
 * normalizeArray, minus the mean, normalizeArray again; mean and (K-1) std of
 * the result. pixels must hold sred_block_size_3d(bw, bh, bd) floats. */
sred_status sred_reference_block_3d(const float *block_vol, int bw, int bh, int bd, float *pixels,
                                    int *block_size, float *mean, float *std_dev);

/* Replaces CLUtils.getLocalStatistics3D (java/CLUtils.java:1030-1131) and
 * cl/kernelGetLocalStatistics3D.cl: per-voxel ellipsoid-block mean and (K-1)
 * standard deviation in FP32, reference evaluation order; border voxels 0. */
sred_status sred_local_statistics_3d(sred_ctx *ctx, const float *vol, int w, int h, int d, int bw, int bh,
                                     int bd, float *means, float *stds);

/* Replaces Utils.getRelevanceMask3D (java/Utils.java:1501-1525) with
 * getMeanNoiseVar3D (java/Utils.java:1463-1498): the noise variance is the
 * mean local variance over the interior (FP32 raster-order sum, float count);
 * mask = 1 where the interior voxel's local variance exceeds
 * noise_var * relevance_constant, else 0. */
sred_status sred_relevance_mask_3d(sred_ctx *ctx, int w, int h, int d, int bw, int bh, int bd,
                                   const float *local_stds, float relevance_constant, float *mask,
                                   float *noise_var);

/* Replaces CLUtils.calculateBlockRepetitionMap3D (java/CLUtils.java:1639-1653)
 * and the four getBlock*3D methods it dispatches to (:1133-1637) with their
 * kernels (cl/kernelGetBlock{Pearson,Ssim,Nrmse,AbsDiffStds}3D.cl), for a
 * volume already prepared by getInputImage3D. metric: "Pearson's R",
 * "SSIM", "NRMSE (inverted)" or "Abs. Diff. of StdDevs."
 * (java/BlockRepetition3D_.java:19-24). FP32 in the kernels' order; then, over
 * the interior, NRMSE inverted (0 -> 1) and Abs-diff as 1 - x, the relevance
 * mask applied when relevance_constant > 0, and normalizeImage3D over the
 * interior (over the mask when one is applied). The Pearson command of the
 * reference passes the block depth as the z radius (java/CLUtils.java:1149,
 * gathering from a box twice as deep); here every metric uses the block's own
 * radius, as the other three do. */
sred_status sred_calculate_block_repetition_map_3d(sred_ctx *ctx, const char *metric, const float *vol, int w,
                                                   int h, int d, const float *ref_pixels, int block_size, int bw,
                                                   int bh, int bd, float ref_mean, float ref_std,
                                                   float relevance_constant, int normalize_output, float *out);

/* Device-resident variant: d_vol and d_out are w*h*d floats on the context's
 * device; runs on `stream` (NULL = the context's stream). */
sred_status sred_block_map_3d_device(sred_ctx *ctx, const char *metric, const float *d_vol, int w, int h, int d,
                                     const float *ref_pixels, int block_size, int bw, int bh, int bd,
                                     float ref_mean, float ref_std, float relevance_constant,
                                     int normalize_output, float *d_out, void *stream);

/* Replaces CLUtils.calculateGlobalRepetitionMap3D (java/CLUtils.java:2793-2816)
 * and the four getGlobal*3D methods (:2225-2790) with their kernels
 * (cl/kernelGetGlobal{Pearson,Ssim,Nrmse,AbsDiffStds}3D.cl), after the
 * preprocessing of java/GlobalRepetition3D_.java:97-143 (local statistics,
 * relevance mask, nPixels). metric: "Pearson's R", "SSIM", "NRMSE" or
 * "Abs. diff. of StdDevs". For every interior voxel p of non-zero local
 * variance with sigma_p^2 >= threshold: num_p = sum over the test voxels q
 * (interior, sigma_q^2 >= threshold; Abs-diff also sigma_q^2 != 0) of
 * term(p, q) w(p, q), den_p = sum of w(p, q), w = exp(-(sigma_p - sigma_q)^2 /
 * (noise_var + eps)); term: Pearson max(0, r), SSIM the kernel's SSIM (the
 * product mu_p^2 mu_q^2 in its denominator), NRMSE the root mean squared
 * difference of the centred blocks, Abs-diff |sigma_p - sigma_q|; a flat test
 * block gives Pearson and SSIM 0. The map is num / (den nPixels + eps), NRMSE
 * and Abs-diff inverted where the mask is 1, the mask applied when
 * relevance_constant > 0, normalizeImage3D over the mask. Sums in FP64 from
 * FP32 terms (the tensor-core engine computes the block dot products in split
 * BF16, as the 2D global map). Repairs of the reference, which does not run as
 * shipped: the relevance mask is getRelevanceMask3D's (noise variance = mean
 * local variance over the interior; the command passes the 2D mask,
 * java/GlobalRepetition3D_.java:126-128, whose indexing fails on the first
 * interior slice), the reference block spans all bd slices (the kernels gather
 * one slice short, e.g. cl/kernelGetGlobalPearson3D.cl:46), and SSIM compiles
 * (cl/kernelGetGlobalSsim3D.cl:76). K <= 512. */
sred_status sred_calculate_global_repetition_map_3d(sred_ctx *ctx, const char *metric, const float *vol, int w,
                                                    int h, int d, int bw, int bh, int bd,
                                                    float relevance_constant, int normalize_output, float *out,
                                                    sred_run_info *info);

/* Device-resident variant of sred_calculate_global_repetition_map_3d. */
sred_status sred_global_map_3d_device(sred_ctx *ctx, const char *metric, const float *d_vol, int w, int h, int d,
                                      int bw, int bh, int bd, float relevance_constant, int normalize_output,
                                      float *d_out, void *stream, sred_run_info *info);

/* ---------------------------------------------------------------------
 * Relevance-mask tools. The image is the one the ImageJ commands compute on:
 * already variance-stabilised (sred_gat_2d) and min-max normalised (the
 * commands normalise in FP64, java/RelevanceMask2D_.java). The block is the
 * ellipse of bw x bh; the commands read the dialog's width and height into
 * each other's radius (java/RelevanceMask2D_.java, bRW = bH / 2), which for a
 * non-square block makes their kernel overrun its patch array, so only square
 * blocks are comparable. Threshold: noise_var * c, or c when the noise
 * variance is 0. A pixel is relevant (1) iff it is interior and s^2 is
 * neither below the threshold nor 0.
 * --------------------------------------------------------------------- */

/* Replaces RelevanceMask2D_.run after its preprocessing: s = the local
 * standard deviation (cl/kernelGetLocalMeans.cl), noise variance from 8x8 or
 * 16x16 tiles with FP64 sums (its getMeanAndVarBlock). mask: w*h floats. */
sred_status sred_relevance_mask_tool_2d(sred_ctx *ctx, const float *img, int w, int h, int bw, int bh,
                                        float filter_constant, float *mask, float *threshold, float *noise_var);

/* Replaces RelevanceMaskStack2D_.run after its preprocessing: n masks at the
 * constants lower, lower + step, ... (FP32 accumulation; the command makes
 * n = ceil((upper - lower) / step) + 1), s = the local variance
 * (cl/kernelGetRelevanceMask2D.cl; the Java code squares it), noise variance
 * from tiles with FP32 sums (OptimiseRelevanceMask_.getRelevanceMap).
 * masks: n*w*h floats, constants: n floats; 1 <= n <= 65535. */
sred_status sred_relevance_mask_sweep_2d(sred_ctx *ctx, const float *img, int w, int h, int bw, int bh, float lower,
                                         float step, int n, float *masks, float *constants, float *noise_var);

/* Replaces OptimiseRelevanceMask_.run after its preprocessing: steps the
 * constant from 0 by `step` (FP32 accumulation) until the mask is all 0 and
 * returns that constant (all_zeros) and the last one whose interior was all 1
 * (all_ones, 0 if none); s and the noise variance as for the sweep. A step
 * that stops increasing the constant is SRED_ERR_ARG (the reference loops
 * forever). */
sred_status sred_relevance_constant_range_2d(sred_ctx *ctx, const float *img, int w, int h, int bw, int bh,
                                             float step, float *all_ones, float *all_zeros, float *noise_var);

/* Replaces ClassifyRedundancy_.run (java/ClassifyRedundancy_.java) on a
 * repetition map: the pixels inside `border` clustered by value into k classes
 * with k-means++ and Lloyd iterations, as its clusterer (commons-math3 3.6.1
 * KMeansPlusPlusClusterer: at most 1000 rounds, an empty cluster refilled with
 * a random point of the cluster whose distances vary most); with optimal_k the
 * elbow of getOptimalK picks k in 1..max_k first (the first k whose WCSS does
 * not fall ends the search). out (w*h floats): the class of each interior
 * pixel ranked by class size (0 = largest, ties in cluster order), border 0.
 * Random choices come from java.util.Random seeded with `seed` (the reference
 * seeds from the clock, a new generator per clustering; one generator serves
 * every clustering of a call here). k_used and wcss (sum of squared distances
 * to the class centres) may be NULL. Classes: 1..64. */
sred_status sred_classify_redundancy_2d(sred_ctx *ctx, const float *map, int w, int h, int border, int k,
                                        int optimal_k, int max_k, int64_t seed, float *out, int *k_used,
                                        double *wcss);

/* Diagnostics (no counterpart in the reference): out[i] = a[i] / b computed
 * on the device the way the 3D Pearson block kernel divides by a shared
 * divisor (Markstein's correction of a * RN(1/b)); equal to IEEE division. */
sred_status sred_debug_divide_fixed(sred_ctx *ctx, const float *a, size_t n, float b, float *out);
/* The same in FP64 (the block-map Hu kernel's divisor: one per block). */
sred_status sred_debug_divide_fixed64(sred_ctx *ctx, const double *a, size_t n, double b, double *out);

/* Variance stabilisation by the quadtree (2D) / octree (3D) method, the
 * "Quad/Octree" option (java/QuadTree_.java, java/OcTree_.java; the commands'
 * defaults and java/Utils.java:686-705 use min_size 4, alpha 0.01, max_iter
 * 50, lts_fraction 0.75). The image is split recursively into quadrants
 * (octants) while a node is larger than min_size along every axis and the
 * Fisher test finds its variance different from the variance of its
 * Laplacian pseudo-residuals (ratio of the smaller to the larger below the
 * alpha quantile of F(n-1, n-1); n = width*height, in 3D too); every leaf
 * gives a robust (Gaussian-weighted) mean and a least-trimmed-squares
 * variance; a least-squares line through the (mean, variance) pairs gives g0
 * (slope) and eDC (intercept), and every pixel is transformed in place as
 * applyGATtree does ((g0 v + 3/8 g0^2 + eDC) < 0 -> 0, else (2/g0) sqrt(...)).
 * Statistics are FP64 sums on the device (the reference: FP32), the F
 * quantiles host FP64 (the reference: commons-math3 FDistribution). In 3D all
 * w*h*d voxels are transformed (the reference's Utils call transforms the
 * first w*h). SRED_ERR_ARG if the regression has no slope. */
sred_status sred_gat_quadtree_2d(sred_ctx *ctx, float *img, int w, int h, int min_size, float alpha, int max_iter,
                                 float lts_fraction, double *g0, double *edc, int *n_leaves);
sred_status sred_gat_octree_3d(sred_ctx *ctx, float *vol, int w, int h, int d, int min_size, float alpha,
                               int max_iter, float lts_fraction, double *g0, double *edc, int *n_leaves);

/* Quantile at p of the F distribution with (df, df) degrees of freedom, the
 * threshold of the trees' Fisher test (host only; NaN outside 0 < p < 1,
 * df > 0). */
double sred_f_quantile(double p, double df);

/* Sharded 3D global map (no counterpart in the reference): the two phases
 * of sred_global_map_2d_shard_sums / _finish for sred_global_map_3d_device;
 * the sums layout and the work-item split are the same ([num | den] over the
 * relevant non-zero-variance blocks). Either finish function completes
 * either map. */
sred_status sred_global_map_3d_shard_sums(sred_ctx *ctx, const char *metric, const float *d_vol, int w, int h, int d,
                                          int bw, int bh, int bd, float relevance_constant, int shard, int n_shards,
                                          double *d_sums, size_t capacity, void *stream, sred_run_info *info);
sred_status sred_global_map_3d_shard_finish(sred_ctx *ctx, const double *d_sums, int normalize_output,
                                            float *d_out, void *stream, sred_run_info *info);

#ifdef __cplusplus
}
#endif
#endif /* SRED_H */
