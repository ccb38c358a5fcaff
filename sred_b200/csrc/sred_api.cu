// libsred C ABI: context, workspaces and the orchestration of the global and
// block repetition maps (the part of java/CLUtils.java and java/Utils.java
// that runs between the plugin commands and the kernels).
#include <algorithm>
#include <cfloat>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "shape.cuh"
#include "cluster.cuh"
#include "gat_tree.cuh"
#include "relevance.cuh"
#include "volume.cuh"

using namespace sred;

namespace {

enum BufId {
  B_IMG, B_MEANS, B_STDS, B_MASK, B_MASKIN, B_FLAGS, B_SLOT, B_GPIX, B_FPIX, B_COUNTS, B_U, B_A, B_B,
  B_PARAMS, B_RMAX, B_NUM, B_DEN, B_SUMS, B_OUT, B_VARS, B_MM, B_NMASK, B_BAD, B_STATUS, B_STDS2, B_COLSOA,
  B_FEAT, B_SIG, B_FR, B_FI, B_GAT, B_OFF3, B_REF3, B_STAT, B_THR, B_KMX, B_KMD2, B_KMLAB, B_KMB, B_TBOX, B_TSTAT, B_TMEAN, B_TVAR, B_STKIN, B_STKOUT,
  B_NBUF
};

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

// A prepared global map: moments, relevance mask, compaction and the
// contraction operands are in the context's workspaces. Kept in the context
// between the two phases of the row-sharded entry points.
struct GState {
  bool valid = false;
  bool vol = false;  // a 3D map (depth d, z radius rd)
  int d = 1, rd = 0;
  int metric = 0, w = 0, h = 0, rw = 0, rh = 0, K = 0, n_g = 0, n_flat = 0, engine = 0, kp = 0, kq = 0;
  size_t n = 0, n_pad = 0;
  float nv = 0, thr = 0, npx = 0, relc = 0;
  bool given = false;
};

}  // namespace

struct sred_ctx {
  int device = 0;
  int num_sms = 148;
  int engine = SRED_ENGINE_FP32;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_in = nullptr, copy_out = nullptr;  // sred_block_map_2d_stack's copy streams (lazily)
  cudaEvent_t ev[6] = {};
  DevBuf buf[B_NBUF];
  std::vector<float> hvars;
  std::string err;
  std::recursive_mutex mu;
  std::vector<sred_ctx*> workers;  // extra contexts of sred_global_map_2d_batch (own streams and workspaces)
  GState shard;                    // the map prepared by sred_global_map_2d_shard_sums
  TcDebug tc_debug{0, -1};         // tensor-core wait limit and withheld tile (sred_debug_set_tc_wait)
  bool tune = false;               // time the launch shapes of an untuned (K', metric, size class)
  void (*log_cb)(const char*, void*) = nullptr;
  void* log_user = nullptr;
};

namespace {

// Host-side fault injection for tests: SRED_FAULT=alloc|launch makes the
// library report that failure without touching the GPU.
bool fault(const char* what) {
  const char* f = std::getenv("SRED_FAULT");
  return f && std::strcmp(f, what) == 0;
}

// Launch-shape tuner of the tensor-core engine, shared by every context of
// the process: (K', metric, size class of the contracted block count) ->
// the fastest shape timed on a map of that key (TcChoice) and its time.
struct TuneKey {
  int kq, metric, nclass;
  bool operator<(const TuneKey& o) const {
    return kq != o.kq ? kq < o.kq : metric != o.metric ? metric < o.metric : nclass < o.nclass;
  }
};
struct TuneEntry {
  TcChoice choice;
  float ms;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneEntry> g_tune;

// Size classes: up to 64 Ki blocks, up to 256 Ki, larger.
int tune_nclass(int n) { return n < (1 << 16) ? 0 : n < (1 << 18) ? 1 : 2; }

// Contraction engine and K' of a global map: Abs-diff needs no contraction
// (the FP32 engine's kernel without a Gram); the other metrics run on the
// context's engine, the tensor cores while the operands' B tile fits in
// shared memory (NRMSE with the three-level split), else the FP32 engine.
int pick_engine(const sred_ctx* c, int metric, int K, int* kq) {
  *kq = split_cols_for(metric, K);
  if (metric == kAbsDiff || c->engine != SRED_ENGINE_TC) return SRED_ENGINE_FP32;
  TcPlan plan;
  return plan_gram_tc(*kq, &plan) ? SRED_ENGINE_TC : SRED_ENGINE_FP32;
}

void log_msg(sred_ctx* c, const std::string& msg) {
  if (c && c->log_cb) c->log_cb(msg.c_str(), c->log_user);
}

sred_status fail(sred_ctx* c, sred_status s, const std::string& msg) {
  if (c) {
    c->err = msg;
    log_msg(c, std::string("error: ") + msg);
  }
  return s;
}

sred_status cuda_fail(sred_ctx* c, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  return fail(c, e == cudaErrorMemoryAllocation ? SRED_ERR_OOM : SRED_ERR_LAUNCH, m);
}

#define CK(call)                                              \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return cuda_fail(c, _e, #call);    \
  } while (0)

#define CKS(expr)                      \
  do {                                 \
    sred_status _s = (expr);           \
    if (_s != SRED_OK) return _s;      \
  } while (0)

template <class T>
sred_status ensure(sred_ctx* c, int id, size_t count, T** out) {
  size_t bytes = std::max<size_t>(count * sizeof(T), 256);
  DevBuf& b = c->buf[id];
  if (fault("alloc")) return fail(c, SRED_ERR_OOM, "injected allocation failure");
  if (b.cap < bytes) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t cap = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&b.p, cap);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc");
    b.cap = cap;
  }
  *out = static_cast<T*>(b.p);
  return SRED_OK;
}

int global_metric(const char* m) {
  if (!m) return -1;
  if (!std::strcmp(m, "Pearson's R")) return kPearson;
  if (!std::strcmp(m, "SSIM")) return kSsim;
  if (!std::strcmp(m, "NRMSE")) return kNrmse;
  if (!std::strcmp(m, "Abs. diff. of StdDevs")) return kAbsDiff;
  return -1;
}

int block_metric(const char* m) {
  if (!m) return -1;
  if (!std::strcmp(m, "Pearson's R")) return kPearson;
  if (!std::strcmp(m, "SSIM")) return kSsim;
  if (!std::strcmp(m, "NRMSE (inverted)")) return kNrmse;
  if (!std::strcmp(m, "Abs. Diff. of StdDevs.")) return kAbsDiff;
  if (!std::strcmp(m, "Cosine")) return kCosine;
  if (!std::strcmp(m, "Hu moments")) return kHu;
  if (!std::strcmp(m, "Phase correlation")) return kPhase;
  if (!std::strcmp(m, "Hu distance")) return kHu7;
  return -1;
}

// nPixels accumulates 1.0f per masked pixel in FP32
// (java/GlobalRepetition2D_.java:133-140), which saturates at 2^24.
float java_float_count(unsigned long long n) { return n <= 16777216ull ? (float)n : 16777216.0f; }

size_t round_up(size_t a, size_t b) { return (a + b - 1) / b * b; }

int grid_for(size_t n, int threads, int cap) {
  size_t g = (n + threads - 1) / threads;
  return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)cap));
}

sred_status check_block(sred_ctx* c, int w, int h, int bw, int bh, Ellipse* e) {
  if (w <= 0 || h <= 0) return fail(c, SRED_ERR_ARG, "image dimensions must be positive");
  if (bw % 2 == 0 || bh % 2 == 0 || bw < 3 || bh < 3)
    return fail(c, SRED_ERR_ARG, "block dimensions must be odd and at least 3");
  int k = build_ellipse(bw, bh, e);
  if (k < 2 || k > kMaxK) return fail(c, SRED_ERR_ARG, "ellipse block size out of range");
  return SRED_OK;
}

// Noise variance, java/Utils.java:790-837: tile variances on the device in
// the reference's FP32 order, then the sort and the mean of the lowest 3% on
// the host in FP32, exactly as the reference does them.
sred_status noise_var_dev(sred_ctx* c, const float* d_img, int w, int h, cudaStream_t st, float* out) {
  const int wh = w * h;
  const int t = (wh <= 352 * 288) ? 8 : 16;
  const int nbx = w / t, nby = h / t, nb = nbx * nby;
  const int nv = (int)(0.03f * (float)nb + 1.0f);
  if (nv > nb) return fail(c, SRED_ERR_ARG, "image smaller than one noise-variance tile");
  float* d_vars;
  int* d_bad;
  CKS(ensure(c, B_VARS, nb, &d_vars));
  CKS(ensure(c, B_BAD, 1, &d_bad));
  CK(cudaMemsetAsync(d_bad, 0, sizeof(int), st));
  k_noise_tiles<<<grid_for(nb, 128, 1 << 30), 128, 0, st>>>(d_img, w, t, nbx, nb, d_vars, d_bad);
  CK(cudaGetLastError());
  c->hvars.resize(nb);
  int bad = 0;
  CK(cudaMemcpyAsync(c->hvars.data(), d_vars, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (bad) return fail(c, SRED_ERR_INVALID_INPUT, "Input contains invalid (NaN or Infinite) values.");
  std::sort(c->hvars.begin(), c->hvars.end());
  float v = 0.0f;
  for (int i = 0; i < nv; i++) v += c->hvars[i];
  v = std::fabs(v / (float)nv);
  v = (1.0f + 0.001f * (v - 40.0f)) * v;
  *out = v;
  return SRED_OK;
}

sred_status normalize_dev(sred_ctx* c, float* d_a, const float* d_mask, int w, int h, int rw, int rh, int planes,
                          cudaStream_t st) {
  unsigned* mm;
  CKS(ensure(c, B_MM, 2 * planes, &mm));
  k_init_minmax<<<grid_for((size_t)planes, 256, 64), 256, 0, st>>>(mm, planes);
  dim3 g(grid_for((size_t)w * h, 256, 4 * c->num_sms), planes);
  k_minmax<<<g, 256, 0, st>>>(d_a, d_mask, w, h, rw, rh, (size_t)w * h, mm);
  k_remap<<<g, 256, 0, st>>>(d_a, d_mask, w, h, rw, rh, (size_t)w * h, mm);
  CK(cudaGetLastError());
  return SRED_OK;
}

struct GivenStats {
  const float* means;  // host
  const float* stds;
  const float* mask;
  float threshold, noise_var, n_pixels;
};


// Phase 1: everything before the all-pairs contraction.
sred_status global_prepare(sred_ctx* c, int metric, const float* d_img, int w, int h, int bw, int bh, float relc,
                           cudaStream_t st, const GivenStats* given, GState* gs) {
  gs->valid = false;
  c->shard.valid = false;  // the workspaces are about to be overwritten
  Ellipse e;
  CKS(check_block(c, w, h, bw, bh, &e));
  const int K = e.k, rw = e.rw, rh = e.rh;
  const size_t n = (size_t)w * h;
  if (n > (size_t)INT32_MAX / 2) return fail(c, SRED_ERR_ARG, "image too large");
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  CK(cudaEventRecord(c->ev[0], st));

  float *d_means, *d_stds, *d_mask;
  CKS(ensure(c, B_MEANS, n, &d_means));
  CKS(ensure(c, B_STDS, n, &d_stds));
  CKS(ensure(c, B_MASK, n, &d_mask));
  float nv, thr;
  const float* d_mask_in = nullptr;
  if (!given) {
    k_local_stats<<<dim3((w + 127) / 128, h), 128, 0, st>>>(d_img, w, h, e, d_means, d_stds);
    CK(cudaGetLastError());
    CKS(noise_var_dev(c, d_img, w, h, st, &nv));
    thr = nv * relc;
  } else {
    float* d_mi;
    CKS(ensure(c, B_MASKIN, n, &d_mi));
    CK(cudaMemcpyAsync(d_means, given->means, n * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_stds, given->stds, n * sizeof(float), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_mi, given->mask, n * sizeof(float), cudaMemcpyHostToDevice, st));
    d_mask_in = d_mi;
    nv = given->noise_var;
    thr = given->threshold;
  }

  uint8_t* d_flags;
  int *d_slot, *d_gpix, *d_fpix;
  int2* d_counts;
  unsigned long long* d_nmask;
  const int nseg = (int)((n + kCompactSeg - 1) / kCompactSeg);
  CKS(ensure(c, B_FLAGS, n, &d_flags));
  CKS(ensure(c, B_SLOT, n, &d_slot));
  CKS(ensure(c, B_GPIX, n, &d_gpix));
  CKS(ensure(c, B_FPIX, n, &d_fpix));
  CKS(ensure(c, B_COUNTS, nseg + 1, &d_counts));
  CKS(ensure(c, B_NMASK, 1, &d_nmask));
  CK(cudaMemsetAsync(d_nmask, 0, sizeof(unsigned long long), st));
  k_flags<<<grid_for(n, 256, 1 << 30), 256, 0, st>>>(d_stds, d_mask_in, w, h, rw, rh, thr, d_mask, d_flags,
                                                      d_nmask);
  k_count<<<nseg, 256, 0, st>>>(d_flags, n, d_counts);
  k_scan<<<1, 1024, 0, st>>>(d_counts, nseg);
  k_scatter<<<nseg, 256, 0, st>>>(d_flags, n, d_counts, d_gpix, d_fpix, d_slot);
  CK(cudaGetLastError());
  int2 tot;
  unsigned long long nmask = 0;
  CK(cudaMemcpyAsync(&tot, d_counts + nseg, sizeof(int2), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&nmask, d_nmask, sizeof(nmask), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const int n_g = tot.x, n_flat = tot.y;
  const float npx = given ? given->n_pixels : java_float_count(nmask);

  // Operands and per-block parameters of the all-pairs contraction.
  int kq;  // K' of the split-BF16 operands
  const int engine = pick_engine(c, metric, K, &kq);
  const size_t n_pad = round_up((size_t)std::max(n_g, 1), 256);
  const int kp = (int)round_up(K, 4);
  float* d_U = nullptr;
  __nv_bfloat16 *d_A = nullptr, *d_B = nullptr;
  BlockParams* d_params;
  float* d_rmax;
  double *d_num, *d_den, *d_sums;
  CKS(ensure(c, B_PARAMS, n_pad, &d_params));
  CKS(ensure(c, B_RMAX, n_pad / 128, &d_rmax));
  CKS(ensure(c, B_NUM, n_pad, &d_num));
  CKS(ensure(c, B_DEN, n_pad, &d_den));
  CKS(ensure(c, B_SUMS, 4, &d_sums));
  if (engine == SRED_ENGINE_FP32 || metric == kNrmse) {  // tensor-core NRMSE reads U for near-identical pairs
    CKS(ensure(c, B_U, n_pad * kp, &d_U));
    CK(cudaMemsetAsync(d_U + (size_t)n_g * kp, 0, (n_pad - n_g) * kp * sizeof(float), st));
  }
  if (engine == SRED_ENGINE_TC) {
    CKS(ensure(c, B_A, n_pad * kq, &d_A));
    CKS(ensure(c, B_B, n_pad * kq, &d_B));
    CK(cudaMemsetAsync(d_A + (size_t)n_g * kq, 0, (n_pad - n_g) * kq * sizeof(__nv_bfloat16), st));
    CK(cudaMemsetAsync(d_B + (size_t)n_g * kq, 0, (n_pad - n_g) * kq * sizeof(__nv_bfloat16), st));
  }
  CK(cudaMemsetAsync(d_params + n_g, 0, (n_pad - n_g) * sizeof(BlockParams), st));
  CK(cudaMemsetAsync(d_rmax, 0, (n_pad / 128) * sizeof(float), st));
  CK(cudaMemsetAsync(d_num, 0, n_pad * sizeof(double), st));
  CK(cudaMemsetAsync(d_den, 0, n_pad * sizeof(double), st));
  CK(cudaMemsetAsync(d_sums, 0, 4 * sizeof(double), st));
  // weight = exp(-(s_p - s_q)^2 / (FILTER_PARAM + EPSILON)) = 2^-(a_p - a_q)^2,
  // FILTER_PARAM + EPSILON summed in FP32 as the reference kernel does.
  const float hden = nv + kEps;
  const float wscale = (float)std::sqrt(1.4426950408889634 / (double)hden);
  if (n_g > 0) {
    // one warp per group of 32 blocks
    const int pgrid = grid_for(((size_t)n_g + 31) / 32 * 32, 256, 8 * c->num_sms);
    const int mode = engine == SRED_ENGINE_FP32 ? 0 : split_levels_for(metric, K) - 1;
    k_pack<<<pgrid, 256, 0, st>>>(d_img, w, e, d_gpix, n_g, wscale, mode, d_U, kp, d_A, d_B, kq, d_params,
                                  d_rmax, d_sums);
    CK(cudaGetLastError());
  }
  if (engine == SRED_ENGINE_TC) {
    float* d_soa;
    CKS(ensure(c, B_COLSOA, gram_tc_soa_floats((int)n_pad), &d_soa));
  }
  CK(cudaEventRecord(c->ev[1], st));
  gs->metric = metric;
  gs->w = w;
  gs->h = h;
  gs->rw = rw;
  gs->rh = rh;
  gs->K = K;
  gs->n_g = n_g;
  gs->n_flat = n_flat;
  gs->engine = engine;
  gs->kp = kp;
  gs->kq = kq;
  gs->n = n;
  gs->n_pad = n_pad;
  gs->nv = nv;
  gs->thr = thr;
  gs->npx = npx;
  gs->relc = relc;
  gs->given = given != nullptr;
  gs->valid = true;
  return SRED_OK;
}

// Phase 2: the all-pairs contraction (work-item range `shard` of n_shards of
// the upper triangle) into the num/den workspaces.
sred_status global_gram(sred_ctx* c, const GState& gs, cudaStream_t st, int shard, int n_shards) {
  if (gs.n_g > 0) {
    EpiConsts ec;
    ec.metric = gs.metric;
    // NRMSE on the FP32 engine accumulates |u_p - u_q|^2 (difference form)
    if (gs.engine == SRED_ENGINE_FP32 && ec.metric == kNrmse) ec.metric = kNrmseD;
    else if (gs.engine == SRED_ENGINE_FP32 && ec.metric == kNrmseW) ec.metric = kNrmseDW;
    ec.n = gs.n_g;
    ec.nrmse_scale = (float)((double)(gs.K - 1) / (double)gs.K);
    ec.c1 = kC1;
    ec.c2 = kC2;
    if (gs.engine == SRED_ENGINE_TC && nrmse_metric(ec.metric)) {
      ec.U = static_cast<const float*>(c->buf[B_U].p);
      ec.kp = gs.kp;
      ec.K = gs.K;
      ec.nrmse_near = kNrmseNear;
    }
    double* d_num = static_cast<double*>(c->buf[B_NUM].p);
    double* d_den = static_cast<double*>(c->buf[B_DEN].p);
    const BlockParams* d_params = static_cast<const BlockParams*>(c->buf[B_PARAMS].p);
    const float* d_rmax = static_cast<const float*>(c->buf[B_RMAX].p);
    if (gs.engine == SRED_ENGINE_FP32) {
      CK(launch_gram_fp32(static_cast<const float*>(c->buf[B_U].p), gs.kp, d_params, d_rmax, ec, d_num, d_den,
                          c->num_sms, st, shard, n_shards));
    } else {
      int* d_status;
      CKS(ensure(c, B_STATUS, 4, &d_status));
      auto run = [&](const TcChoice* ch) -> sred_status {
        CK(cudaMemsetAsync(d_status, 0, 4 * sizeof(int), st));
        CK(launch_gram_tc(static_cast<const __nv_bfloat16*>(c->buf[B_A].p),
                          static_cast<const __nv_bfloat16*>(c->buf[B_B].p), gs.kq, (int)gs.n_pad, d_params,
                          static_cast<float*>(c->buf[B_COLSOA].p), ec, d_num, d_den, c->num_sms, d_status, st, shard,
                          n_shards, &c->tc_debug, ch));
        return SRED_OK;
      };
      // The tuned shape of this key (sharded maps keep the default shape, so
      // that every shard partitions the work alike).
      TcChoice chosen;
      bool have = false;
      const TuneKey key{gs.kq, ec.metric, tune_nclass(gs.n_g)};
      if (n_shards == 1) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto f = g_tune.find(key);
        if (f != g_tune.end()) {
          chosen = f->second.choice;
          have = true;
        }
      }
      if (!have && c->tune && n_shards == 1) {
        // time every shape that fits on this map's operands (each from zeroed
        // sums), keep the fastest, then compute the map with it. Maps running
        // on other streams at the same time perturb these timings, so a
        // tuning pass is best run on one context at a time.
        TcChoice cand[16];
        const int nc = gram_tc_candidates(gs.kq, cand, 16);
        float best = 3.4e38f;
        for (int i = 0; i < nc; i++) {
          CK(cudaMemsetAsync(d_num, 0, gs.n_pad * sizeof(double), st));
          CK(cudaMemsetAsync(d_den, 0, gs.n_pad * sizeof(double), st));
          CK(cudaEventRecord(c->ev[4], st));
          CKS(run(&cand[i]));
          CK(cudaEventRecord(c->ev[5], st));
          CK(cudaEventSynchronize(c->ev[5]));
          float ms = 0.0f;
          CK(cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]));
          if (ms < best) {
            best = ms;
            chosen = cand[i];
          }
        }
        if (nc > 0) {
          have = true;
          std::lock_guard<std::mutex> lk(g_tune_mu);
          g_tune[key] = TuneEntry{chosen, best};
        }
        CK(cudaMemsetAsync(d_num, 0, gs.n_pad * sizeof(double), st));
        CK(cudaMemsetAsync(d_den, 0, gs.n_pad * sizeof(double), st));
        CK(cudaEventRecord(c->ev[1], st));  // ms_gram times the map's own contraction, not the tuning
      }
      CKS(run(have ? &chosen : nullptr));
      int status = 0;
      CK(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (status) return fail(c, SRED_ERR_TIMEOUT, "tensor-core pipeline wait exceeded its bound");
    }
  }
  CK(cudaEventRecord(c->ev[2], st));
  return SRED_OK;
}

// Phase 3: per-pixel finalisation (num / (den nPixels + eps), inversion,
// mask), normalisation, run info.
sred_status global_finish(sred_ctx* c, const GState& gs, cudaStream_t st, int normalize, float* d_out,
                          sred_run_info* info) {
  const double sk = std::sqrt((double)(gs.K - 1) / (double)gs.K);
  const float* d_mask = static_cast<const float*>(c->buf[B_MASK].p);
  k_finalize<<<grid_for(gs.n, 256, 1 << 30), 256, 0, st>>>(
      static_cast<const int*>(c->buf[B_SLOT].p), gs.w, gs.h, gs.rw, gs.rh,
      static_cast<const double*>(c->buf[B_NUM].p), static_cast<const double*>(c->buf[B_DEN].p),
      static_cast<const BlockParams*>(c->buf[B_PARAMS].p), static_cast<const double*>(c->buf[B_SUMS].p),
      gs.n_flat, gs.metric, sk, (double)gs.npx, d_mask, gs.relc > 0.0f ? 1 : 0, d_out);
  CK(cudaGetLastError());
  if (normalize) CKS(normalize_dev(c, d_out, d_mask, gs.w, gs.h, gs.rw, gs.rh, 1, st));
  CK(cudaEventRecord(c->ev[3], st));
  CK(cudaEventSynchronize(c->ev[3]));
  if (info) {
    info->n_blocks = (int64_t)std::max(0, gs.w - 2 * gs.rw) * std::max(0, gs.h - 2 * gs.rh);
    info->n_relevant = (int64_t)gs.n_g + gs.n_flat;
    info->n_flat = gs.n_flat;
    info->pairs = (double)info->n_relevant * (double)info->n_relevant;
    info->noise_var = gs.nv;
    info->threshold = gs.thr;
    info->n_pixels = gs.npx;
    info->k = gs.K;
    info->engine = gs.engine;
    float t01 = 0, t12 = 0, t23 = 0, t03 = 0;
    cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&t12, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]);
    cudaEventElapsedTime(&t03, c->ev[0], c->ev[3]);
    info->ms_moments = t01;
    info->ms_gram = t12;
    info->ms_finalize = t23;
    info->ms_total = t03;
    info->launches = (gs.given ? 0 : 2) + 4 + (gs.n_g > 0 ? (gs.engine == SRED_ENGINE_TC ? 3 : 2) : 0) + 1 +
                     (normalize ? 3 : 0);
  }
  if (c->log_cb) {
    float t03 = 0;
    cudaEventElapsedTime(&t03, c->ev[0], c->ev[3]);
    char line[256];
    std::snprintf(line, sizeof(line), "global map %dx%d K=%d: %d relevant blocks (%d flat), %s engine, %.3f ms",
                  gs.w, gs.h, gs.K, gs.n_g + gs.n_flat, gs.n_flat,
                  gs.engine == SRED_ENGINE_TC ? "tensor-core" : "fp32", t03);
    log_msg(c, line);
  }
  return SRED_OK;
}

// The global repetition map on device-resident data.
sred_status global_core(sred_ctx* c, int metric, const float* d_img, int w, int h, int bw, int bh, float relc,
                        int normalize, float* d_out, cudaStream_t st, sred_run_info* info,
                        const GivenStats* given) {
  GState gs;
  CKS(global_prepare(c, metric, d_img, w, h, bw, bh, relc, st, given, &gs));
  CKS(global_gram(c, gs, st, 0, 1));
  return global_finish(c, gs, st, normalize, d_out, info);
}

// Raw block map of the shape metrics (stds_out: FP32 local stds, or NULL).
// Hu moments: cl/kernelGetPatchHu2D.cl with the reference block prepared by
// hu_prepare_patch; phase correlation: the block-map form of
// cl/kernelGetPhaseCorrelationMap.cl (k_block_phase).
sred_status block_shape_launch(sred_ctx* c, int metric, const float* d_img, int w, int h, int frames,
                               const Ellipse& e, const float* ref_pixels, int bw, int bh, float ref_std, float* d_out,
                               float* d_stds, cudaStream_t st) {
  const size_t plane = (size_t)w * h;
  const dim3 grid((unsigned)((plane + 127) / 128), (unsigned)frames);
  if (metric == kHu) {
    std::vector<float> patch((size_t)bw * bh);
    hu_prepare_patch(ref_pixels, bw, bh, patch.data());
    k_patch_hu<<<grid, 128, 0, st>>>(d_img, w, h, e, e.k, patch_hu1(patch.data(), bw, bh), d_out, d_stds);
  } else if (metric == kHu7) {
    Hu7Ref r;
    hu7_reference(ref_pixels, e, &r);
    launch_block_hu7(d_img, w, h, frames, e, r, d_out, d_stds, st);
  } else {
    if (bw > kPhaseMaxDim || bh > kPhaseMaxDim)
      return fail(c, SRED_ERR_ARG, "phase correlation supports blocks up to 15x15");
    PhaseRef pr;
    phase_reference_dft(ref_pixels, ref_std, bw, bh, &pr);
    launch_block_phase(d_img, w, h, frames, e, bw, bh, pr, d_out, d_stds, st);
  }
  CK(cudaGetLastError());
  return SRED_OK;
}

sred_status block_core(sred_ctx* c, int metric, const float* d_img, int w, int h, int frames,
                       const float* ref_pixels, int block_size, int bw, int bh, float ref_mean, float ref_std,
                       float relc, int normalize, float* d_out, cudaStream_t st) {
  c->shard.valid = false;  // shares workspaces with the global map
  Ellipse e;
  CKS(check_block(c, w, h, bw, bh, &e));
  if (block_size != e.k) return fail(c, SRED_ERR_ARG, "block_size does not match the ellipse of bw x bh");
  if (frames < 1 || frames > 65535) return fail(c, SRED_ERR_ARG, "frames must be in 1..65535");
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  const int rw = e.rw, rh = e.rh;
  const size_t plane = (size_t)w * h, n = plane * frames;
  RefBlock rb;
  rb.k = e.k;
  rb.mean = ref_mean;
  rb.std = ref_std;
  std::memcpy(rb.px, ref_pixels, sizeof(float) * e.k);
  const bool need_mask = (metric == kNrmse) || relc > 0.0f;
  float* d_stds = nullptr;
  if (need_mask) CKS(ensure(c, B_STDS2, n, &d_stds));
  if (metric == kHu || metric == kHu7 || metric == kPhase) {
    CKS(block_shape_launch(c, metric, d_img, w, h, frames, e, ref_pixels, bw, bh, ref_std, d_out, d_stds, st));
  } else {
    dim3 grid, blk;
    block_map_launch_shape(w, h, frames, &grid, &blk);
    const size_t smem = block_map_smem(e);
    if (smem > 200 * 1024) return fail(c, SRED_ERR_ARG, "block too large for the streaming tile");
    if (smem > 48 * 1024)
      CK(cudaFuncSetAttribute(k_block_map, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_block_map<<<grid, blk, smem, st>>>(d_img, w, h, frames, e, rb, metric, d_out, d_stds);
  }
  CK(cudaGetLastError());

  float* d_mask = nullptr;
  const dim3 pg(grid_for(plane, 256, 4 * c->num_sms), frames);
  auto relevance_masks = [&]() -> sred_status {
    float* d_m;
    uint8_t* d_flags;
    unsigned long long* d_cnt;
    CKS(ensure(c, B_MASK, n, &d_m));
    CKS(ensure(c, B_FLAGS, plane, &d_flags));
    CKS(ensure(c, B_NMASK, 1, &d_cnt));
    for (int f = 0; f < frames; f++) {
      float nv;
      CKS(noise_var_dev(c, d_img + f * plane, w, h, st, &nv));
      k_flags<<<grid_for(plane, 256, 1 << 30), 256, 0, st>>>(d_stds + f * plane, nullptr, w, h, rw, rh,
                                                             nv * relc, d_m + f * plane, d_flags, d_cnt);
    }
    CK(cudaGetLastError());
    d_mask = d_m;
    return SRED_OK;
  };

  if (metric == kNrmse) {
    if (relc == 0.0f) {
      CKS(ensure(c, B_MASK, n, &d_mask));
      k_interior_mask<<<pg, 256, 0, st>>>(d_mask, w, h, rw, rh, plane);
    } else {
      CKS(relevance_masks());
    }
    k_apply_mask<<<grid_for(n, 256, 8 * c->num_sms), 256, 0, st>>>(d_out, d_mask, n);
    CKS(normalize_dev(c, d_out, d_mask, w, h, rw, rh, frames, st));
    k_invert_masked<<<pg, 256, 0, st>>>(d_out, d_mask, w, h, rw, rh, plane);
    if (normalize) CKS(normalize_dev(c, d_out, d_mask, w, h, rw, rh, frames, st));
  } else {
    if (metric == kAbsDiff) {
      unsigned* mm;
      CKS(ensure(c, B_MM, 2 * frames, &mm));
      k_init_minmax<<<grid_for((size_t)frames, 256, 64), 256, 0, st>>>(mm, frames);
      k_minmax<<<pg, 256, 0, st>>>(d_out, nullptr, w, h, rw, rh, plane, mm);
      k_block_absdiff_post<<<pg, 256, 0, st>>>(d_out, w, h, rw, rh, plane, mm);
    }
    if (relc > 0.0f) {
      CKS(relevance_masks());
      k_apply_mask<<<grid_for(n, 256, 8 * c->num_sms), 256, 0, st>>>(d_out, d_mask, n);
    }
    if (normalize) CKS(normalize_dev(c, d_out, d_mask, w, h, rw, rh, frames, st));
  }
  CK(cudaGetLastError());
  return SRED_OK;  // enqueued on st; the callers decide when to wait
}

// ---------------------------------------------------------------------------
// 3D block repetition maps (java/CLUtils.java:1030-1653)
// ---------------------------------------------------------------------------

// Validates a volume and an ellipsoid block and uploads the block offsets.
sred_status prepare_volume(sred_ctx* c, int w, int h, int d, int bw, int bh, int bd, cudaStream_t st, Vol3* v,
                           int** d_off) {
  if (w <= 0 || h <= 0 || d <= 0) return fail(c, SRED_ERR_ARG, "volume dimensions must be positive");
  if (bw % 2 == 0 || bh % 2 == 0 || bd % 2 == 0 || bw < 3 || bh < 3 || bd < 3)
    return fail(c, SRED_ERR_ARG, "block dimensions must be odd and at least 3");
  if ((h + 3) / 4 > 65535 || d > 65535) return fail(c, SRED_ERR_ARG, "volume height or depth too large");
  if ((long long)(bd / 2) * w * h + (long long)(bh / 2) * w + bw / 2 > 0x7fffffffll)
    return fail(c, SRED_ERR_ARG, "block offsets exceed 32 bits");
  std::vector<int> off(kMaxK3);
  const int k = build_ellipsoid(bw, bh, bd, w, h, off.data());
  if (k < 2 || k > kMaxK3) return fail(c, SRED_ERR_ARG, "ellipsoid block size out of range");
  CKS(ensure(c, B_OFF3, k, d_off));
  CK(cudaMemcpyAsync(*d_off, off.data(), sizeof(int) * k, cudaMemcpyHostToDevice, st));
  *v = Vol3{w, h, d, bw / 2, bh / 2, bd / 2, k};
  return SRED_OK;
}

dim3 vol_grid(const Vol3& v) { return dim3((v.W + 31) / 32, (v.H + 3) / 4, v.D); }

// java/Utils.java:1463-1498 (getMeanNoiseVar3D): the mean of the local
// variances over the interior, summed in FP32 in raster order with a float
// count, as the reference does on the host.
float noise_var_3d(const Vol3& v, const float* stds) {
  float s = 0.0f, n = 0.0f;
  for (int z = v.rd; z < v.D - v.rd; z++)
    for (int y = v.rh; y < v.H - v.rh; y++)
      for (int x = v.rw; x < v.W - v.rw; x++) {
        const float sd = stds[((size_t)z * v.H + y) * v.W + x];
        s += sd * sd;
        n += 1.0f;
      }
  return s / n;
}

// Relevance mask of a volume from device local stds (the noise variance on
// the host from a copy of them); map, if not null, is multiplied by the mask.
sred_status mask_3d(sred_ctx* c, const Vol3& v, const float* d_stds, float relc, float* d_mask, float* d_map,
                    cudaStream_t st, float* noise_var) {
  const size_t n = (size_t)v.W * v.H * v.D;
  std::vector<float> h_stds(n);
  CK(cudaMemcpyAsync(h_stds.data(), d_stds, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const float nv = noise_var_3d(v, h_stds.data());
  k_mask3d<<<vol_grid(v), dim3(32, 4), 0, st>>>(d_stds, v, nv * relc, d_mask, d_map);
  CK(cudaGetLastError());
  if (noise_var) *noise_var = nv;
  return SRED_OK;
}

// With h_vol, d_vol is filled from host memory here, in slabs of slices on
// the context's upload stream, and each slab's local statistics and map run
// as soon as the slices they read have landed, so the upload overlaps the
// kernels; the slabs' maps equal one launch over the volume.
sred_status block3d_core(sred_ctx* c, int metric, const float* d_vol, int w, int h, int d, const float* ref_pixels,
                         int block_size, int bw, int bh, int bd, float ref_mean, float ref_std, float relc,
                         int normalize, float* d_out, cudaStream_t st, const float* h_vol = nullptr) {
  c->shard.valid = false;  // shares workspaces with the global map
  if (metric < kPearson || metric > kAbsDiff) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown 3D block metric");
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  Vol3 v;
  int* d_off;
  CKS(prepare_volume(c, w, h, d, bw, bh, bd, st, &v, &d_off));
  if (block_size != v.k) return fail(c, SRED_ERR_ARG, "block_size does not match the ellipsoid of bw x bh x bd");
  const size_t n = (size_t)w * h * d;
  float *d_ref, *d_means, *d_stds;
  CKS(ensure(c, B_REF3, v.k, &d_ref));
  CKS(ensure(c, B_MEANS, n, &d_means));
  CKS(ensure(c, B_STDS, n, &d_stds));
  CK(cudaMemcpyAsync(d_ref, ref_pixels, sizeof(float) * v.k, cudaMemcpyHostToDevice, st));
  const dim3 grid = vol_grid(v), blk(32, 4);
  // slices [z0, z1): local statistics, map, metric transform
  auto slab = [&](int z0, int z1) -> sred_status {
    if (z1 <= z0) return SRED_OK;
    Vol3 vs = v;
    vs.z0 = z0;
    const dim3 gs(grid.x, grid.y, z1 - z0);
    k_local_stats3d<<<gs, blk, sizeof(int) * v.k, st>>>(d_vol, vs, d_off, d_means, d_stds);
    CK(launch_block_map3d(d_vol, vs, d_off, d_ref, ref_mean, ref_std, metric, d_means, d_stds, d_out, st, z1));
    if (metric == kNrmse || metric == kAbsDiff) k_block3d_post<<<gs, blk, 0, st>>>(d_out, vs, metric);
    CK(cudaGetLastError());
    return SRED_OK;
  };
  if (!h_vol) {
    CKS(slab(0, d));
  } else {
    // slabs of about 16 MiB (at most 64): the map of slices [z0, z1) reads
    // slices [z0 - rd, z1 + rd), so after slab i has landed the slices up to
    // its end minus rd are computed
    const size_t plane = (size_t)w * h;
    int ds = (int)std::max<size_t>(1, ((size_t)16 << 20) / (plane * sizeof(float)));
    ds = std::max(ds, (d + 63) / 64);
    const int ns = (d + ds - 1) / ds;
    if (!c->copy_in) CK(cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
    std::vector<cudaEvent_t> up(ns, nullptr);
    sred_status res = SRED_OK;
    cudaError_t e = cudaEventRecord(c->ev[5], st);  // the volume buffer may still be read by earlier work
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_in, c->ev[5], 0);
    int done = 0;  // slices computed so far
    for (int i = 0; i < ns && e == cudaSuccess && res == SRED_OK; i++) {
      const int z_lo = i * ds, z_hi = std::min(d, z_lo + ds);
      e = cudaEventCreateWithFlags(&up[i], cudaEventDisableTiming);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(const_cast<float*>(d_vol) + (size_t)z_lo * plane, h_vol + (size_t)z_lo * plane,
                            (size_t)(z_hi - z_lo) * plane * sizeof(float), cudaMemcpyHostToDevice, c->copy_in);
      if (e == cudaSuccess) e = cudaEventRecord(up[i], c->copy_in);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(st, up[i], 0);
      if (e != cudaSuccess) break;
      const int z_end = i == ns - 1 ? d : std::max(done, z_hi - v.rd);
      res = slab(done, z_end);
      done = z_end;
    }
    cudaStreamSynchronize(c->copy_in);  // the host volume is no longer read
    for (cudaEvent_t x : up)
      if (x) cudaEventDestroy(x);
    if (e != cudaSuccess) return cuda_fail(c, e, "block3d_core: slab upload");
    CKS(res);
  }
  float* d_mask = nullptr;
  if (relc > 0.0f) {
    CKS(ensure(c, B_MASK, n, &d_mask));
    CKS(mask_3d(c, v, d_stds, relc, d_mask, d_out, st, nullptr));
  }
  if (normalize) {
    unsigned* mm;
    CKS(ensure(c, B_MM, 2, &mm));
    k_init_minmax<<<1, 32, 0, st>>>(mm, 1);
    k_minmax3d<<<grid_for((size_t)v.W * v.H * v.D, 256, 4 * c->num_sms), 256, 0, st>>>(d_out, d_mask, v, mm);
    k_remap3d<<<grid, blk, 0, st>>>(d_out, d_mask, v, mm);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

// The 3D global repetition map on a device-resident volume
// (java/GlobalRepetition3D_.java:97-158, java/CLUtils.java:2225-2816): local
// statistics, the relevance mask of getRelevanceMask3D (the command passes
// the 2D mask, which fails on its first interior slice), the compacted block
// lists, the all-pairs contraction on the 2D engines, the 3D host steps.
sred_status global3d_prepare(sred_ctx* c, int metric, const float* d_vol, int w, int h, int d, int bw, int bh,
                             int bd, float relc, cudaStream_t st, GState* gs) {
  gs->valid = false;
  c->shard.valid = false;  // shares workspaces with the 2D global map
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  CK(cudaEventRecord(c->ev[0], st));
  Vol3 v;
  int* d_off;
  CKS(prepare_volume(c, w, h, d, bw, bh, bd, st, &v, &d_off));
  if (v.k > kMaxK) return fail(c, SRED_ERR_ARG, "ellipsoid block size above 512 for the global map");
  const size_t n = (size_t)w * h * d;
  if (n > (size_t)INT32_MAX / 2) return fail(c, SRED_ERR_ARG, "volume too large");
  const int K = v.k;
  float *d_means, *d_stds, *d_mask;
  CKS(ensure(c, B_MEANS, n, &d_means));
  CKS(ensure(c, B_STDS, n, &d_stds));
  CKS(ensure(c, B_MASK, n, &d_mask));
  const dim3 grid = vol_grid(v), blk(32, 4);
  k_local_stats3d<<<grid, blk, sizeof(int) * K, st>>>(d_vol, v, d_off, d_means, d_stds);
  CK(cudaGetLastError());
  std::vector<float> h_stds(n);
  CK(cudaMemcpyAsync(h_stds.data(), d_stds, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const float nv = noise_var_3d(v, h_stds.data());
  const bool has_interior = w > 2 * v.rw && h > 2 * v.rh && d > 2 * v.rd;
  if (has_interior && !std::isfinite(nv))
    return fail(c, SRED_ERR_INVALID_INPUT, "Input contains invalid (NaN or Infinite) values.");
  const float thr = nv * relc;

  uint8_t* d_flags;
  int *d_slot, *d_gpix, *d_fpix;
  int2* d_counts;
  unsigned long long* d_nmask;
  const int nseg = (int)((n + kCompactSeg - 1) / kCompactSeg);
  CKS(ensure(c, B_FLAGS, n, &d_flags));
  CKS(ensure(c, B_SLOT, n, &d_slot));
  CKS(ensure(c, B_GPIX, n, &d_gpix));
  CKS(ensure(c, B_FPIX, n, &d_fpix));
  CKS(ensure(c, B_COUNTS, nseg + 1, &d_counts));
  CKS(ensure(c, B_NMASK, 1, &d_nmask));
  CK(cudaMemsetAsync(d_nmask, 0, sizeof(unsigned long long), st));
  k_flags3d<<<grid_for(n, 256, 4 * c->num_sms), 256, 0, st>>>(d_stds, v, thr, metric == kAbsDiff ? 0 : 1, d_mask,
                                                                d_flags, d_nmask);
  k_count<<<nseg, 256, 0, st>>>(d_flags, n, d_counts);
  k_scan<<<1, 1024, 0, st>>>(d_counts, nseg);
  k_scatter<<<nseg, 256, 0, st>>>(d_flags, n, d_counts, d_gpix, d_fpix, d_slot);
  CK(cudaGetLastError());
  int2 tot;
  unsigned long long nmask = 0;
  CK(cudaMemcpyAsync(&tot, d_counts + nseg, sizeof(int2), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&nmask, d_nmask, sizeof(nmask), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const int n_g = tot.x, n_flat = tot.y;
  const float npx = java_float_count(nmask);

  int kq;
  const int engine = pick_engine(c, metric, K, &kq);
  const size_t n_pad = round_up((size_t)std::max(n_g, 1), 256);
  const int kp = (int)round_up(K, 4);
  float* d_U = nullptr;
  __nv_bfloat16 *d_A = nullptr, *d_B = nullptr;
  BlockParams* d_params;
  float* d_rmax;
  double *d_num, *d_den;
  CKS(ensure(c, B_PARAMS, n_pad, &d_params));
  CKS(ensure(c, B_RMAX, n_pad / 128, &d_rmax));
  CKS(ensure(c, B_NUM, n_pad, &d_num));
  CKS(ensure(c, B_DEN, n_pad, &d_den));
  if (engine == SRED_ENGINE_FP32 || metric == kNrmse) {  // tensor-core NRMSE reads U for near-identical pairs
    CKS(ensure(c, B_U, n_pad * kp, &d_U));
    CK(cudaMemsetAsync(d_U + (size_t)n_g * kp, 0, (n_pad - n_g) * kp * sizeof(float), st));
  }
  if (engine == SRED_ENGINE_TC) {
    CKS(ensure(c, B_A, n_pad * kq, &d_A));
    CKS(ensure(c, B_B, n_pad * kq, &d_B));
    CK(cudaMemsetAsync(d_A + (size_t)n_g * kq, 0, (n_pad - n_g) * kq * sizeof(__nv_bfloat16), st));
    CK(cudaMemsetAsync(d_B + (size_t)n_g * kq, 0, (n_pad - n_g) * kq * sizeof(__nv_bfloat16), st));
  }
  CK(cudaMemsetAsync(d_params + n_g, 0, (n_pad - n_g) * sizeof(BlockParams), st));
  CK(cudaMemsetAsync(d_rmax, 0, (n_pad / 128) * sizeof(float), st));
  CK(cudaMemsetAsync(d_num, 0, n_pad * sizeof(double), st));
  CK(cudaMemsetAsync(d_den, 0, n_pad * sizeof(double), st));
  // weight = exp(-(s_p - s_q)^2 / (FILTER_PARAM + EPSILON)) = 2^-(a_p - a_q)^2
  const float hden = nv + kEps;
  const float wscale = (float)std::sqrt(1.4426950408889634 / (double)hden);
  if (n_g > 0) {
    k_pack3d<<<grid_for((size_t)n_g * 32, 256, 8 * c->num_sms), 256, 0, st>>>(
        d_vol, v, d_off, d_gpix, n_g, wscale, engine == SRED_ENGINE_FP32 ? 0 : split_levels_for(metric, K) - 1, d_U, kp, d_A,
        d_B, kq, d_params, d_rmax);
    CK(cudaGetLastError());
  }
  if (engine == SRED_ENGINE_TC) {
    float* d_soa;
    CKS(ensure(c, B_COLSOA, gram_tc_soa_floats((int)n_pad), &d_soa));
  }
  CK(cudaEventRecord(c->ev[1], st));
  gs->vol = true;
  gs->metric = metric == kNrmse ? kNrmseW : metric;
  gs->w = w;
  gs->h = h;
  gs->d = d;
  gs->rw = v.rw;
  gs->rh = v.rh;
  gs->rd = v.rd;
  gs->K = K;
  gs->n_g = n_g;
  gs->n_flat = n_flat;
  gs->engine = engine;
  gs->kp = kp;
  gs->kq = kq;
  gs->n = n;
  gs->n_pad = n_pad;
  gs->nv = nv;
  gs->thr = thr;
  gs->npx = npx;
  gs->relc = relc;
  gs->valid = true;
  return SRED_OK;
}

// Finalisation of a prepared 3D map whose num/den workspaces hold the sums.
sred_status global3d_finish(sred_ctx* c, const GState& gs, cudaStream_t st, int normalize, float* d_out,
                            sred_run_info* info) {
  const int metric = gs.metric == kNrmseW ? kNrmse : gs.metric;
  const Vol3 v{gs.w, gs.h, gs.d, gs.rw, gs.rh, gs.rd, gs.K};
  const dim3 grid = vol_grid(v), blk(32, 4);
  const float* d_mask = static_cast<const float*>(c->buf[B_MASK].p);
  k_finalize3d<<<grid, blk, 0, st>>>(static_cast<const int*>(c->buf[B_SLOT].p), v,
                                     static_cast<const double*>(c->buf[B_NUM].p),
                                     static_cast<const double*>(c->buf[B_DEN].p),
                                     static_cast<const BlockParams*>(c->buf[B_PARAMS].p), gs.n_flat, metric,
                                     std::sqrt((double)(gs.K - 1) / (double)gs.K), (double)gs.npx, d_mask,
                                     gs.relc > 0.0f ? 1 : 0, d_out);
  CK(cudaGetLastError());
  if (normalize) {
    unsigned* mm;
    CKS(ensure(c, B_MM, 2, &mm));
    k_init_minmax<<<1, 32, 0, st>>>(mm, 1);
    k_minmax3d<<<grid_for((size_t)v.W * v.H * v.D, 256, 4 * c->num_sms), 256, 0, st>>>(d_out, d_mask, v, mm);
    k_remap3d<<<grid, blk, 0, st>>>(d_out, d_mask, v, mm);
    CK(cudaGetLastError());
  }
  CK(cudaEventRecord(c->ev[3], st));
  CK(cudaEventSynchronize(c->ev[3]));
  if (info) {
    info->n_blocks = (int64_t)std::max(0, gs.w - 2 * gs.rw) * std::max(0, gs.h - 2 * gs.rh) *
                     std::max(0, gs.d - 2 * gs.rd);
    info->n_relevant = (int64_t)gs.n_g + gs.n_flat;
    info->n_flat = gs.n_flat;
    info->pairs = (double)gs.n_g * (double)info->n_relevant;
    info->noise_var = gs.nv;
    info->threshold = gs.thr;
    info->n_pixels = gs.npx;
    info->k = gs.K;
    info->engine = gs.engine;
    float t01 = 0, t12 = 0, t23 = 0, t03 = 0;
    cudaEventElapsedTime(&t01, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&t12, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&t23, c->ev[2], c->ev[3]);
    cudaEventElapsedTime(&t03, c->ev[0], c->ev[3]);
    info->ms_moments = t01;
    info->ms_gram = t12;
    info->ms_finalize = t23;
    info->ms_total = t03;
    info->launches = 5 + (gs.n_g > 0 ? (gs.engine == SRED_ENGINE_TC ? 3 : 2) : 0) + 1 + (normalize ? 3 : 0);
  }
  if (c->log_cb) {
    float t03 = 0;
    cudaEventElapsedTime(&t03, c->ev[0], c->ev[3]);
    char line[256];
    std::snprintf(line, sizeof(line),
                  "global map %dx%dx%d K=%d: %d reference blocks, %d flat test blocks, %s engine, %.3f ms", gs.w,
                  gs.h, gs.d, gs.K, gs.n_g, gs.n_flat, gs.engine == SRED_ENGINE_TC ? "tensor-core" : "fp32", t03);
    log_msg(c, line);
  }
  return SRED_OK;
}

sred_status global3d_core(sred_ctx* c, int metric, const float* d_vol, int w, int h, int d, int bw, int bh, int bd,
                          float relc, int normalize, float* d_out, cudaStream_t st, sred_run_info* info) {
  GState gs;
  CKS(global3d_prepare(c, metric, d_vol, w, h, d, bw, bh, bd, relc, st, &gs));
  CKS(global_gram(c, gs, st, 0, 1));
  return global3d_finish(c, gs, st, normalize, d_out, info);
}

// ---------------------------------------------------------------------------
// Relevance-mask tools (java/RelevanceMask2D_.java, RelevanceMaskStack2D_.java,
// OptimiseRelevanceMask_.java)
// ---------------------------------------------------------------------------

// The tools' noise variance: t x t tile variances (t = 8 up to CIF size, else
// 16), FP32 sums (OptimiseRelevanceMask_.getMeanAndVarBlock) or FP64 sums
// (RelevanceMask2D_.getMeanAndVarBlock), sorted, the mean of the lowest 3% in
// FP32, then (1 + 0.001 (v - 40)) v. No NaN check (the tools have none).
sred_status tool_noise_var(sred_ctx* c, const float* d_img, int w, int h, bool fp64, cudaStream_t st, float* out) {
  const int wh = w * h;
  const int t = (wh <= 352 * 288) ? 8 : 16;
  const int nbx = w / t, nby = h / t, nb = nbx * nby;
  const int nv = (int)(0.03f * (float)nb + 1.0f);
  if (nv > nb) return fail(c, SRED_ERR_ARG, "image smaller than one noise-variance tile");
  float* d_vars;
  int* d_bad;
  CKS(ensure(c, B_VARS, nb, &d_vars));
  CKS(ensure(c, B_BAD, 1, &d_bad));
  if (fp64) {
    k_noise_tiles64<<<grid_for(nb, 128, 1 << 30), 128, 0, st>>>(d_img, w, t, nbx, nb, d_vars);
  } else {
    k_noise_tiles<<<grid_for(nb, 128, 1 << 30), 128, 0, st>>>(d_img, w, t, nbx, nb, d_vars, d_bad);
  }
  CK(cudaGetLastError());
  c->hvars.resize(nb);
  CK(cudaMemcpyAsync(c->hvars.data(), d_vars, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::sort(c->hvars.begin(), c->hvars.end());
  float v = 0.0f;
  for (int i = 0; i < nv; i++) v += c->hvars[i];
  v = std::fabs(v / (float)nv);
  *out = (1.0f + 0.001f * (v - 40.0f)) * v;
  return SRED_OK;
}

// Uploads the image and computes the tools' block statistic (local std or
// local variance) into B_STAT.
sred_status tool_stat(sred_ctx* c, const float* img, int w, int h, int bw, int bh, int take_sqrt, Ellipse* e,
                      float** d_img_out, float** d_stat_out) {
  CKS(check_block(c, w, h, bw, bh, e));
  const size_t n = (size_t)w * h;
  float *d_img, *d_stat;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_STAT, n, &d_stat));
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  k_local_var2d<<<dim3((w + 127) / 128, h), 128, 0, c->stream>>>(d_img, w, h, *e, take_sqrt, d_stat);
  CK(cudaGetLastError());
  *d_img_out = d_img;
  *d_stat_out = d_stat;
  return SRED_OK;
}

// Threshold of the tools: noise_var * c, or c itself when the noise variance is 0.
float tool_threshold(float nv, float c) { return nv == 0.0f ? c : nv * c; }

sred_status tool_masks(sred_ctx* c, const float* d_stat, int w, int h, const Ellipse& e, const float* thr, int n,
                       float* masks) {
  float *d_thr, *d_masks;
  const size_t px = (size_t)w * h;
  // at most 256 MiB of masks on the device at a time
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n, ((size_t)64 << 20) / px));
  CKS(ensure(c, B_THR, n, &d_thr));
  CKS(ensure(c, B_OUT, px * chunk, &d_masks));
  CK(cudaMemcpyAsync(d_thr, thr, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
  for (int i0 = 0; i0 < n; i0 += chunk) {
    const int m = std::min(chunk, n - i0);
    k_sweep_masks<<<dim3(grid_for(px, 256, 2 * c->num_sms), m), 256, 0, c->stream>>>(d_stat, w, h, e.rw, e.rh,
                                                                                       d_thr + i0, d_masks);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(masks + px * i0, d_masks, px * m * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// Redundancy classification (java/ClassifyRedundancy_.java)
// ---------------------------------------------------------------------------

// java.util.Random (48-bit linear congruential generator), the generator of
// the clusterer (commons-math3 JDKRandomGenerator): nextInt(bound) and
// nextDouble() as the JDK defines them.
struct JavaRandom {
  uint64_t seed;
  explicit JavaRandom(int64_t s) : seed(((uint64_t)s ^ 0x5DEECE66DULL) & ((1ULL << 48) - 1)) {}
  int next(int bits) {
    seed = (seed * 0x5DEECE66DULL + 0xBULL) & ((1ULL << 48) - 1);
    return (int)(int64_t)(seed >> (48 - bits));
  }
  int next_int(int bound) {
    if ((bound & -bound) == bound) return (int)(((int64_t)bound * (int64_t)next(31)) >> 31);
    int bits, val;
    do {
      bits = next(31);
      val = bits % bound;
    } while ((int64_t)bits - val + (bound - 1) > INT32_MAX);
    return val;
  }
  double next_double() { return (double)(((int64_t)next(26) << 27) + next(27)) * 0x1.0p-53; }
};

struct KmState {
  size_t n = 0;
  int nblk = 0;
  double *x = nullptr, *d2 = nullptr, *blk = nullptr;
  int* lab = nullptr;
  unsigned long long* changed = nullptr;
};

// One clustering: k-means++ centres, then Lloyd until no point changes
// cluster (and no cluster was refilled) or 1000 rounds. Returns the centres,
// the per-cluster counts and the WCSS; labels stay in st.lab.
sred_status kmeans_run(sred_ctx* c, KmState& st, int k, JavaRandom& rng, std::vector<double>& centers,
                       std::vector<double>& counts, double* wcss) {
  cudaStream_t s = c->stream;
  const size_t n = st.n;
  const int nb = st.nblk;
  std::vector<double> part(nb);
  std::vector<size_t> taken;
  centers.assign(k, 0.0);
  // first centre: a uniformly chosen point
  size_t first = (size_t)rng.next_int((int)n);
  double xv;
  CK(cudaMemcpyAsync(&xv, st.x + first, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  centers[0] = xv;
  taken.push_back(first);
  int have = 1;
  while (have < k) {
    k_km_d2<<<nb, kKmThreads, 0, s>>>(st.x, n, centers[have - 1], have == 1, st.d2, st.blk);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(part.data(), st.blk, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    double sum = 0.0;
    for (int b = 0; b < nb; b++) sum += part[b];
    const double r = rng.next_double() * sum;
    // the first point whose running sum of d^2 reaches r: whole blocks, then
    // the points of that block in index order
    size_t pick = SIZE_MAX;
    double run = 0.0;
    for (int b = 0; b < nb && pick == SIZE_MAX; b++) {
      if (run + part[b] < r && b + 1 < nb) {
        run += part[b];
        continue;
      }
      const size_t i0 = (size_t)b * kKmSpan, i1 = std::min(n, i0 + kKmSpan);
      std::vector<double> d(i1 - i0);
      CK(cudaMemcpyAsync(d.data(), st.d2 + i0, sizeof(double) * d.size(), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (size_t i = i0; i < i1; i++) {
        run += d[i - i0];
        if (run >= r && std::find(taken.begin(), taken.end(), i) == taken.end()) {
          pick = i;
          break;
        }
      }
      if (pick == SIZE_MAX && run >= r) {
        // rounding left r above this block's running sum: its last untaken point
        for (size_t i = i1; i-- > i0;)
          if (std::find(taken.begin(), taken.end(), i) == taken.end()) {
            pick = i;
            break;
          }
      }
    }
    if (pick == SIZE_MAX) {  // every remaining weight is 0: the last untaken point
      for (size_t i = n; i-- > 0;)
        if (std::find(taken.begin(), taken.end(), i) == taken.end()) {
          pick = i;
          break;
        }
    }
    if (pick == SIZE_MAX) break;
    CK(cudaMemcpyAsync(&xv, st.x + pick, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    centers[have++] = xv;
    taken.push_back(pick);
  }
  k = have;
  centers.resize(k);
  double *d_c, *bsum, *bcnt, *bw;
  CKS(ensure(c, B_KMB, (size_t)nb * (2 * k + 1) + k, &bsum));
  bcnt = bsum + (size_t)nb * k;
  bw = bcnt + (size_t)nb * k;
  d_c = bw + nb;
  std::vector<double> hs((size_t)nb * k), hc((size_t)nb * k), hw(nb);
  CK(cudaMemsetAsync(st.lab, 0xff, n * sizeof(int), s));  // -1: every point counts as changed
  auto assign = [&](unsigned long long* changes) -> sred_status {
    CK(cudaMemcpyAsync(d_c, centers.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(st.changed, 0, sizeof(unsigned long long), s));
    k_km_assign<<<nb, kKmThreads, 0, s>>>(st.x, n, d_c, k, st.lab, st.changed, bsum, bcnt, bw);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hs.data(), bsum, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hc.data(), bcnt, sizeof(double) * hc.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hw.data(), bw, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(changes, st.changed, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return SRED_OK;
  };
  auto cluster_sums = [&](std::vector<double>& sum, std::vector<double>& cnt) {
    sum.assign(k, 0.0);
    cnt.assign(k, 0.0);
    for (int b = 0; b < nb; b++)
      for (int j = 0; j < k; j++) {
        sum[j] += hs[(size_t)b * k + j];
        cnt[j] += hc[(size_t)b * k + j];
      }
  };
  unsigned long long changes = 0;
  CKS(assign(&changes));
  std::vector<double> sum, cnt;
  for (int it = 0; it < 1000; it++) {
    cluster_sums(sum, cnt);
    bool empty = false;
    std::vector<double> next(k);
    for (int j = 0; j < k; j++)
      if (cnt[j] > 0.0) next[j] = sum[j] / cnt[j];
    for (int j = 0; j < k; j++) {
      if (cnt[j] > 0.0) continue;
      // empty: a random point of the cluster whose distances to its centre
      // vary most (sample variance; 0 for a single point)
      empty = true;
      double* d1 = bsum;  // reuse: [nb][k] sums of |d| and of d^2
      double* d2s = bcnt;
      CK(cudaMemcpyAsync(d_c, centers.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
      k_km_distvar<<<nb, kKmThreads, 0, s>>>(st.x, n, d_c, k, st.lab, d1, d2s);
      CK(cudaGetLastError());
      std::vector<double> a((size_t)nb * k), b2((size_t)nb * k);
      CK(cudaMemcpyAsync(a.data(), d1, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(b2.data(), d2s, sizeof(double) * b2.size(), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      int sel = -1;
      double best = -HUGE_VAL;
      for (int q = 0; q < k; q++) {
        if (!(cnt[q] > 0.0)) continue;
        double s1 = 0.0, s2 = 0.0;
        for (int bb = 0; bb < nb; bb++) {
          s1 += a[(size_t)bb * k + q];
          s2 += b2[(size_t)bb * k + q];
        }
        const double var = cnt[q] > 1.0 ? (s2 - s1 * s1 / cnt[q]) / (cnt[q] - 1.0) : 0.0;
        if (var > best) {
          best = var;
          sel = q;
        }
      }
      if (sel < 0) return fail(c, SRED_ERR_INTERNAL, "k-means: no cluster to refill from");
      const int want = rng.next_int((int)cnt[sel]);
      std::vector<int> labs(n);
      CK(cudaMemcpyAsync(labs.data(), st.lab, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      int seen = 0;
      for (size_t i = 0; i < n; i++)
        if (labs[i] == sel && seen++ == want) {
          CK(cudaMemcpyAsync(&xv, st.x + i, sizeof(double), cudaMemcpyDeviceToHost, s));
          CK(cudaStreamSynchronize(s));
          next[j] = xv;
          cnt[sel] -= 1.0;
          break;
        }
    }
    centers = next;
    CKS(assign(&changes));
    if (changes == 0 && !empty) break;
  }
  cluster_sums(sum, cnt);
  counts = cnt;
  double w = 0.0;
  for (int b = 0; b < nb; b++) w += hw[b];
  *wcss = w;
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// Quadtree / octree variance stabilisation (java/QuadTree_.java, OcTree_.java)
// ---------------------------------------------------------------------------

// Regularised incomplete beta I_x(a, b) by the continued fraction of
// Numerical Recipes (Press et al., 3rd ed., section 6.4: the fraction
// evaluated with the modified Lentz method, Lentz 1976), with the symmetry
// I_x(a, b) = 1 - I_{1-x}(b, a) where the fraction converges slowly.
double beta_cf(double a, double b, double x) {
  const double fpmin = 1e-300, eps = 1e-16;
  const double qab = a + b, qap = a + 1.0, qam = a - 1.0;
  double c = 1.0, d = 1.0 - qab * x / qap;
  if (std::fabs(d) < fpmin) d = fpmin;
  d = 1.0 / d;
  double h = d;
  for (int m = 1; m <= 1000000; m++) {
    const int m2 = 2 * m;
    double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
    d = 1.0 + aa * d;
    if (std::fabs(d) < fpmin) d = fpmin;
    c = 1.0 + aa / c;
    if (std::fabs(c) < fpmin) c = fpmin;
    d = 1.0 / d;
    h *= d * c;
    aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
    d = 1.0 + aa * d;
    if (std::fabs(d) < fpmin) d = fpmin;
    c = 1.0 + aa / c;
    if (std::fabs(c) < fpmin) c = fpmin;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (std::fabs(del - 1.0) < eps) break;
  }
  return h;
}

double reg_inc_beta(double a, double b, double x) {
  if (x <= 0.0) return 0.0;
  if (x >= 1.0) return 1.0;
  const double front = std::exp(std::lgamma(a + b) - std::lgamma(a) - std::lgamma(b) + a * std::log(x) +
                                b * std::log1p(-x));
  if (x < (a + 1.0) / (a + b + 2.0)) return front * beta_cf(a, b, x) / a;
  return 1.0 - front * beta_cf(b, a, 1.0 - x) / b;
}

// Quantile at p of the F distribution with (df, df) degrees of freedom: X ~
// F(df, df) iff X / (1 + X) ~ Beta(df/2, df/2); the Beta quantile by
// bisection of I_x(df/2, df/2) to the last bit.
double f_quantile_equal_df(double p, double df) {
  const double a = 0.5 * df;
  double lo = 0.0, hi = 1.0;
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (reg_inc_beta(a, a, mid) < p) lo = mid;
    else hi = mid;
  }
  const double x = 0.5 * (lo + hi);
  return x / (1.0 - x);
}

// The Fisher test of the reference (QuadTree_.performFisherTest): split when
// min(var)/max(var) < F^-1(alpha; n - 1, n - 1), the quantile as float.
bool fisher_split(double var_z, double var_e, int64_t region, float alpha, std::vector<std::pair<int64_t, float>>& cache) {
  const float vz = (float)var_z, ve = (float)var_e;
  const float ratio = std::min(vz, ve) / std::max(vz, ve);
  const int64_t df = region - 1;
  if (df < 1) return false;
  float thr = 0.0f;
  bool found = false;
  for (auto& e : cache)
    if (e.first == df) {
      thr = e.second;
      found = true;
      break;
    }
  if (!found) {
    thr = (float)f_quantile_equal_df((double)alpha, (double)df);
    cache.emplace_back(df, thr);
  }
  return ratio < thr;
}

// Least-squares line through (mean, variance) pairs, updated point by point
// as commons-math3's SimpleRegression does (centred sums with the running
// means; slope = Sxy / Sxx, intercept = (sum y - slope sum x) / n).
void simple_regression(const std::vector<double>& xs, const std::vector<double>& ys, double* slope, double* icpt) {
  double sx = 0, sy = 0, sxx = 0, sxy = 0, xbar = 0, ybar = 0;
  for (size_t i = 0; i < xs.size(); i++) {
    const double x = xs[i], y = ys[i];
    if (i == 0) {
      xbar = x;
      ybar = y;
    } else {
      const double n = (double)i, f1 = 1.0 + n, f2 = n / (1.0 + n);
      const double dx = x - xbar, dy = y - ybar;
      sxx += dx * dx * f2;
      sxy += dx * dy * f2;
      xbar += dx / f1;
      ybar += dy / f1;
    }
    sx += x;
    sy += y;
  }
  const double n = (double)xs.size();
  *slope = (n < 2 || std::fabs(sxx) < 10 * DBL_MIN) ? std::nan("") : sxy / sxx;
  *icpt = (sy - *slope * sx) / n;
}

// The tree of QuadTree_ / OcTree_ built level by level (every level's split
// criteria in one launch), then the robust mean and LTS variance of every
// leaf (one launch each), the regression of the leaves' variances on their
// means in the reference's leaf order (depth first, children in the order
// the reference creates them), and the transform with its slope and
// intercept. d_img holds the image (w x h x d) on the device.
sred_status gat_tree_core(sred_ctx* c, float* d_img, int w, int h, int d, bool octree, int min_size, float alpha,
                          int max_iter, float frac, double* g0_out, double* edc_out, int* n_leaves) {
  if (min_size < 1 || !(alpha > 0.0f && alpha < 1.0f) || max_iter < 1 || !(frac > 0.0f && frac <= 1.0f))
    return fail(c, SRED_ERR_ARG, "tree GAT: min_size >= 1, 0 < alpha < 1, max_iter >= 1, 0 < fraction <= 1");
  cudaStream_t st = c->stream;
  const float l = octree ? 7.0f : 5.0f;
  const float scale = (float)(1.0 / std::sqrt((double)(l * l + l)));
  struct Node {
    TreeBox b;
    int first_child;  // -1: leaf
  };
  std::vector<Node> nodes{{{0, 0, 0, w, h, d}, -1}};
  std::vector<int> level{0};
  std::vector<std::pair<int64_t, float>> fcache;
  const int nch = octree ? 8 : 4;
  while (!level.empty()) {
    // nodes the size test lets split: only their criterion matters
    std::vector<int> cand;
    for (int i : level) {
      const TreeBox& b = nodes[i].b;
      if (!(b.w <= min_size || b.h <= min_size || (octree && b.d <= min_size))) cand.push_back(i);
    }
    std::vector<int> next;
    if (!cand.empty()) {
      TreeBox* d_boxes;
      double* d_stats;
      CKS(ensure(c, B_TBOX, cand.size(), &d_boxes));
      CKS(ensure(c, B_TSTAT, 2 * cand.size(), &d_stats));
      std::vector<TreeBox> hb(cand.size());
      for (size_t j = 0; j < cand.size(); j++) hb[j] = nodes[cand[j]].b;
      CK(cudaMemcpyAsync(d_boxes, hb.data(), sizeof(TreeBox) * hb.size(), cudaMemcpyHostToDevice, st));
      k_tree_node_stats<<<(unsigned)cand.size(), kTreeThreads, 0, st>>>(d_img, w, h, d, d_boxes, octree ? 1 : 0,
                                                                         scale, d_stats);
      CK(cudaGetLastError());
      std::vector<double> hs(2 * cand.size());
      CK(cudaMemcpyAsync(hs.data(), d_stats, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      for (size_t j = 0; j < cand.size(); j++) {
        const TreeBox b = nodes[cand[j]].b;
        // the reference's degrees of freedom: width * height - 1, in 3D too
        if (!fisher_split(hs[2 * j], hs[2 * j + 1], (int64_t)b.w * b.h, alpha, fcache)) continue;
        const int hw = b.w / 2, hh = b.h / 2, hd = octree ? b.d / 2 : 1;
        nodes[cand[j]].first_child = (int)nodes.size();
        for (int k = 0; k < nch; k++) {
          const int ox = (k & 1) ? hw : 0, oy = (k & 2) ? hh : 0, oz = (k & 4) ? hd : 0;
          nodes.push_back({{b.x + ox, b.y + oy, b.z + oz, hw, hh, hd}, -1});
          next.push_back((int)nodes.size() - 1);
        }
      }
    }
    level.swap(next);
  }
  // leaves in the reference's traversal order
  std::vector<TreeBox> leaves;
  std::vector<int> stack{0};
  while (!stack.empty()) {
    const int i = stack.back();
    stack.pop_back();
    if (nodes[i].first_child < 0) {
      leaves.push_back(nodes[i].b);
    } else {
      for (int k = nch - 1; k >= 0; k--) stack.push_back(nodes[i].first_child + k);
    }
  }
  const size_t nl = leaves.size();
  TreeBox* d_boxes;
  float *d_means, *d_vars;
  CKS(ensure(c, B_TBOX, nl, &d_boxes));
  CKS(ensure(c, B_TMEAN, nl, &d_means));
  CKS(ensure(c, B_TVAR, nl, &d_vars));
  CK(cudaMemcpyAsync(d_boxes, leaves.data(), sizeof(TreeBox) * nl, cudaMemcpyHostToDevice, st));
  k_tree_robust_mean<<<(unsigned)nl, kTreeThreads, 0, st>>>(d_img, w, h, d_boxes, max_iter, d_means);
  k_tree_lts<<<(unsigned)nl, kTreeThreads, 0, st>>>(d_img, w, h, d_boxes, d_means, frac, d_vars);
  CK(cudaGetLastError());
  std::vector<float> hm(nl), hv(nl);
  CK(cudaMemcpyAsync(hm.data(), d_means, sizeof(float) * nl, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(hv.data(), d_vars, sizeof(float) * nl, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::vector<double> xs(nl), ys(nl);
  for (size_t i = 0; i < nl; i++) {
    xs[i] = hm[i];
    ys[i] = hv[i];
  }
  double g0, edc;
  simple_regression(xs, ys, &g0, &edc);
  if (!std::isfinite(g0) || g0 == 0.0) return fail(c, SRED_ERR_ARG, "tree GAT: the regression has no slope");
  // applyGATtree: refConstant = 3/8 g0^2 + eDC; (g0 v + c) < 0 -> 0
  const size_t n = (size_t)w * h * d;
  k_gat<<<grid_for(n, 256, 8 * c->num_sms), 256, 0, st>>>(d_img, n, g0, 0.375 * g0 * g0 + edc);
  CK(cudaGetLastError());
  *g0_out = g0;
  *edc_out = edc;
  if (n_leaves) *n_leaves = (int)nl;
  return SRED_OK;
}

cudaStream_t pick(sred_ctx* c, void* s) { return s ? (cudaStream_t)s : c->stream; }

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* sred_status_string(sred_status s) {
  switch (s) {
    case SRED_OK: return "ok";
    case SRED_ERR_ARG: return "invalid argument";
    case SRED_ERR_UNKNOWN_METRIC: return "unknown metric";
    case SRED_ERR_NODEV: return "no CUDA device";
    case SRED_ERR_OOM: return "out of device memory";
    case SRED_ERR_LAUNCH: return "kernel launch or CUDA call failed";
    case SRED_ERR_TIMEOUT: return "device wait timed out";
    case SRED_ERR_INTERNAL: return "internal error";
    case SRED_ERR_INVALID_INPUT: return "input contains NaN or Inf";
  }
  return "unknown status";
}

const char* sred_last_error(sred_ctx* c) { return c ? c->err.c_str() : ""; }

int sred_block_size(int bw, int bh) {
  if (bw < 3 || bh < 3) return 0;
  Ellipse e;
  int k = build_ellipse(bw, bh, &e);
  return k;
}

sred_status sred_create(int device, sred_ctx** out) {
  if (!out) return SRED_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return SRED_ERR_NODEV;
  }
  if (device < 0 || device >= ndev) return SRED_ERR_NODEV;
  sred_ctx* c = new sred_ctx();
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { delete c; return SRED_ERR_NODEV; }
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return SRED_ERR_LAUNCH; }
  for (auto& e : c->ev) cudaEventCreate(&e);
  *out = c;
  return SRED_OK;
}

sred_status sred_destroy(sred_ctx* c) {
  if (!c) return SRED_ERR_ARG;
  for (sred_ctx* w : c->workers) sred_destroy(w);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& b : c->buf)
    if (b.p) cudaFree(b.p);
  for (auto& e : c->ev) cudaEventDestroy(e);
  if (c->copy_in) cudaStreamDestroy(c->copy_in);
  if (c->copy_out) cudaStreamDestroy(c->copy_out);
  cudaStreamDestroy(c->stream);
  delete c;
  return SRED_OK;
}

sred_status sred_set_log_callback(sred_ctx* c, void (*cb)(const char* message, void* user), void* user) {
  if (!c) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->log_cb = cb;
  c->log_user = user;
  return SRED_OK;
}

sred_status sred_set_engine(sred_ctx* c, int engine) {
  if (!c || (engine != SRED_ENGINE_TC && engine != SRED_ENGINE_FP32)) return SRED_ERR_ARG;
  c->engine = engine;
  return SRED_OK;
}

sred_status sred_local_statistics_2d(sred_ctx* c, const float* img, int w, int h, int bw, int bh,
                                     float* means, float* stds) {
  if (!c || !img || !means || !stds) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  Ellipse e;
  CKS(check_block(c, w, h, bw, bh, &e));
  const size_t n = (size_t)w * h;
  float *d_img, *d_m, *d_s;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_MEANS, n, &d_m));
  CKS(ensure(c, B_STDS, n, &d_s));
  cudaStream_t st = c->stream;
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, st));
  k_local_stats<<<dim3((w + 127) / 128, h), 128, 0, st>>>(d_img, w, h, e, d_m, d_s);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(means, d_m, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(stds, d_s, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

sred_status sred_mean_noise_var_2d(sred_ctx* c, const float* img, int w, int h, float* noise_var) {
  if (!c || !img || !noise_var || w <= 0 || h <= 0) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const size_t n = (size_t)w * h;
  float* d_img;
  CKS(ensure(c, B_IMG, n, &d_img));
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  return noise_var_dev(c, d_img, w, h, c->stream, noise_var);
}

sred_status sred_relevance_mask_2d(sred_ctx* c, const float* img, int w, int h, int bw, int bh,
                                   const float* stds, float relc, float* mask, float* threshold, float* noise_var) {
  if (!c || !img || !stds || !mask || !threshold || !noise_var) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->shard.valid = false;  // overwrites workspaces of a prepared shard
  cudaSetDevice(c->device);
  if (w <= 0 || h <= 0 || bw < 1 || bh < 1) return fail(c, SRED_ERR_ARG, "bad dimensions");
  const size_t n = (size_t)w * h;
  float *d_img, *d_s, *d_m;
  uint8_t* d_f;
  unsigned long long* d_cnt;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_STDS, n, &d_s));
  CKS(ensure(c, B_MASK, n, &d_m));
  CKS(ensure(c, B_FLAGS, n, &d_f));
  CKS(ensure(c, B_NMASK, 1, &d_cnt));
  cudaStream_t st = c->stream;
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_s, stds, n * sizeof(float), cudaMemcpyHostToDevice, st));
  float nv;
  CKS(noise_var_dev(c, d_img, w, h, st, &nv));
  const float thr = nv * relc;
  k_flags<<<grid_for(n, 256, 1 << 30), 256, 0, st>>>(d_s, nullptr, w, h, bw / 2, bh / 2, thr, d_m, d_f, d_cnt);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(mask, d_m, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *threshold = thr;
  *noise_var = nv;
  return SRED_OK;
}

sred_status sred_calculate_global_repetition_map_2d(sred_ctx* c, const char* metric, const float* img, int w,
                                                    int h, int bw, int bh, int block_size,
                                                    const float* local_means, const float* local_stds,
                                                    const float* mask, float relc, float threshold,
                                                    float noise_var, float n_pixels, int normalize, float* out,
                                                    sred_run_info* info) {
  if (!c || !img || !local_means || !local_stds || !mask || !out) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (block_size != sred_block_size(bw, bh))
    return fail(c, SRED_ERR_ARG, "block_size does not match the ellipse of bw x bh");
  const size_t n = (size_t)w * h;
  if (w <= 0 || h <= 0) return fail(c, SRED_ERR_ARG, "bad dimensions");
  float *d_img, *d_out;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_OUT, n, &d_out));
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  GivenStats g{local_means, local_stds, mask, threshold, noise_var, n_pixels};
  CKS(global_core(c, m, d_img, w, h, bw, bh, relc, normalize, d_out, c->stream, info, &g));
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_global_map_2d(sred_ctx* c, const char* metric, const float* img, int w, int h, int bw, int bh,
                               float relc, int normalize, float* out, sred_run_info* info) {
  if (!c || !img || !out) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (w <= 0 || h <= 0) return fail(c, SRED_ERR_ARG, "bad dimensions");
  const size_t n = (size_t)w * h;
  float *d_img, *d_out;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_OUT, n, &d_out));
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CKS(global_core(c, m, d_img, w, h, bw, bh, relc, normalize, d_out, c->stream, info, nullptr));
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

// Grows a context's global-map workspaces to the largest of `jobs` (upper
// bounds: every interior block relevant), so that no job reallocates, and
// thereby synchronises the device, while other workers' kernels run.
sred_status reserve_global(sred_ctx* c, const sred_job* jobs, int n_jobs) {
  size_t n = 1, n_pad = 256, a = 1, u = 1, cols = 1;
  bool fp32 = c->engine == SRED_ENGINE_FP32, tc = c->engine == SRED_ENGINE_TC;
  for (int i = 0; i < n_jobs; i++) {
    const sred_job& j = jobs[i];
    Ellipse e;
    if (j.w <= 0 || j.h <= 0 || j.bw < 3 || j.bh < 3 || j.bw % 2 == 0 || j.bh % 2 == 0) continue;
    const int K = build_ellipse(j.bw, j.bh, &e);
    if (K < 2 || K > kMaxK) continue;
    const size_t inter = (size_t)std::max(0, j.w - 2 * e.rw) * std::max(0, j.h - 2 * e.rh);
    const size_t np = round_up(std::max<size_t>(inter, 1), 256);
    n = std::max(n, (size_t)j.w * j.h);
    n_pad = std::max(n_pad, np);
    a = std::max(a, np * (size_t)split_cols_for(global_metric(j.metric), K));
    u = std::max(u, np * round_up(K, 4));
    cols = std::max(cols, gram_tc_soa_floats((int)np));
    int kq;
    if (tc && pick_engine(c, global_metric(j.metric), K, &kq) == SRED_ENGINE_FP32) fp32 = true;
    if (global_metric(j.metric) == kNrmse) fp32 = true;  // U for the near-identical pairs
    if (global_metric(j.metric) == kAbsDiff) fp32 = true;
  }
  float* f;
  uint8_t* u8;
  int* i32;
  int2* i2;
  BlockParams* bp;
  double* d;
  __nv_bfloat16* bf;
  for (int id : {B_IMG, B_OUT, B_MEANS, B_STDS, B_MASK, B_MASKIN}) CKS(ensure(c, id, n, &f));
  CKS(ensure(c, B_FLAGS, n, &u8));
  for (int id : {B_SLOT, B_GPIX, B_FPIX}) CKS(ensure(c, id, n, &i32));
  CKS(ensure(c, B_COUNTS, n / kCompactSeg + 2, &i2));
  CKS(ensure(c, B_PARAMS, n_pad, &bp));
  CKS(ensure(c, B_RMAX, n_pad / 128, &f));
  CKS(ensure(c, B_NUM, n_pad, &d));
  CKS(ensure(c, B_DEN, n_pad, &d));
  if (tc) {
    CKS(ensure(c, B_A, a, &bf));
    CKS(ensure(c, B_B, a, &bf));
    CKS(ensure(c, B_COLSOA, cols, &f));
  }
  if (fp32) CKS(ensure(c, B_U, u, &f));
  return SRED_OK;
}

// Jobs are taken in order from a shared counter by `n_workers` host threads,
// each driving its own context (the caller's and up to seven extra ones kept
// in the caller's context), so one map's host steps and transfers overlap
// another map's kernels. Every map is computed exactly as by
// sred_global_map_2d.
sred_status sred_global_map_2d_batch(sred_ctx* c, sred_job* jobs, int n_jobs, int n_workers) {
  if (!c || n_jobs < 0 || (n_jobs > 0 && !jobs)) return SRED_ERR_ARG;
  if (n_jobs == 0) return SRED_OK;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  n_workers = std::max(1, std::min(n_workers, std::min(8, n_jobs)));
  while ((int)c->workers.size() < n_workers - 1) {
    sred_ctx* w = nullptr;
    const sred_status s = sred_create(c->device, &w);
    if (s != SRED_OK) return fail(c, s, "could not create a batch worker context");
    c->workers.push_back(w);
  }
  for (sred_ctx* w : c->workers) {
    w->engine = c->engine;
    w->tune = c->tune;
  }
  CKS(reserve_global(c, jobs, n_jobs));
  for (int k = 0; k < n_workers - 1; k++) {
    const sred_status s = reserve_global(c->workers[k], jobs, n_jobs);
    if (s != SRED_OK) return fail(c, s, "batch workspace: " + c->workers[k]->err);
  }
  std::atomic<int> next(0);
  auto run = [&](sred_ctx* w) {
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= n_jobs) break;
      sred_job& j = jobs[i];
      j.status = sred_global_map_2d(w, j.metric, j.img, j.w, j.h, j.bw, j.bh, j.relevance_constant,
                                    j.normalize_output, j.out, j.info);
    }
  };
  std::vector<std::thread> threads;
  for (int k = 1; k < n_workers; k++) threads.emplace_back(run, c->workers[k - 1]);
  run(c);
  for (auto& t : threads) t.join();
  for (int i = 0; i < n_jobs; i++)
    if (jobs[i].status != SRED_OK) return fail(c, (sred_status)jobs[i].status, "batch job " + std::to_string(i) + " failed");
  return SRED_OK;
}

sred_status sred_global_map_2d_shard_sums(sred_ctx* c, const char* metric, const float* d_img, int w, int h,
                                          int bw, int bh, float relc, int shard, int n_shards, double* d_sums,
                                          size_t capacity, void* stream, sred_run_info* info) {
  if (!c || !d_img || !d_sums || n_shards < 1 || shard < 0 || shard >= n_shards) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  cudaStream_t st = pick(c, stream);
  GState gs;
  CKS(global_prepare(c, m, d_img, w, h, bw, bh, relc, st, nullptr, &gs));
  if (capacity < 2 * (size_t)gs.n_g) return fail(c, SRED_ERR_ARG, "sums buffer smaller than 2 x relevant blocks");
  CKS(global_gram(c, gs, st, shard, n_shards));
  if (gs.n_g > 0) {
    CK(cudaMemcpyAsync(d_sums, c->buf[B_NUM].p, gs.n_g * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(d_sums + gs.n_g, c->buf[B_DEN].p, gs.n_g * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  CK(cudaStreamSynchronize(st));
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->n_blocks = (int64_t)std::max(0, w - 2 * gs.rw) * std::max(0, h - 2 * gs.rh);
    info->n_relevant = (int64_t)gs.n_g + gs.n_flat;
    info->n_flat = gs.n_flat;
    info->pairs = (double)info->n_relevant * (double)info->n_relevant;
    info->noise_var = gs.nv;
    info->threshold = gs.thr;
    info->n_pixels = gs.npx;
    info->k = gs.K;
    info->engine = gs.engine;
  }
  c->shard = gs;
  return SRED_OK;
}

sred_status sred_global_map_2d_shard_finish(sred_ctx* c, const double* d_sums, int normalize, float* d_out,
                                            void* stream, sred_run_info* info) {
  if (!c || !d_sums || !d_out) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (!c->shard.valid) return fail(c, SRED_ERR_ARG, "no map prepared by a shard_sums call on this context");
  cudaStream_t st = pick(c, stream);
  const GState gs = c->shard;
  c->shard.valid = false;
  if (gs.n_g > 0) {
    CK(cudaMemcpyAsync(c->buf[B_NUM].p, d_sums, gs.n_g * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(c->buf[B_DEN].p, d_sums + gs.n_g, gs.n_g * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  CK(cudaEventRecord(c->ev[0], st));
  CK(cudaEventRecord(c->ev[1], st));
  CK(cudaEventRecord(c->ev[2], st));
  return gs.vol ? global3d_finish(c, gs, st, normalize, d_out, info) : global_finish(c, gs, st, normalize, d_out, info);
}

sred_status sred_global_map_3d_shard_sums(sred_ctx* c, const char* metric, const float* d_vol, int w, int h, int d,
                                          int bw, int bh, int bd, float relc, int shard, int n_shards, double* d_sums,
                                          size_t capacity, void* stream, sred_run_info* info) {
  if (!c || !d_vol || !d_sums || n_shards < 1 || shard < 0 || shard >= n_shards) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  cudaStream_t st = pick(c, stream);
  GState gs;
  CKS(global3d_prepare(c, m, d_vol, w, h, d, bw, bh, bd, relc, st, &gs));
  if (capacity < 2 * (size_t)gs.n_g) return fail(c, SRED_ERR_ARG, "sums buffer smaller than 2 x relevant blocks");
  CKS(global_gram(c, gs, st, shard, n_shards));
  if (gs.n_g > 0) {
    CK(cudaMemcpyAsync(d_sums, c->buf[B_NUM].p, gs.n_g * sizeof(double), cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(d_sums + gs.n_g, c->buf[B_DEN].p, gs.n_g * sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  CK(cudaStreamSynchronize(st));
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->n_blocks = (int64_t)std::max(0, w - 2 * gs.rw) * std::max(0, h - 2 * gs.rh) * std::max(0, d - 2 * gs.rd);
    info->n_relevant = (int64_t)gs.n_g + gs.n_flat;
    info->n_flat = gs.n_flat;
    info->pairs = (double)gs.n_g * (double)info->n_relevant;
    info->noise_var = gs.nv;
    info->threshold = gs.thr;
    info->n_pixels = gs.npx;
    info->k = gs.K;
    info->engine = gs.engine;
  }
  c->shard = gs;
  return SRED_OK;
}

sred_status sred_global_map_3d_shard_finish(sred_ctx* c, const double* d_sums, int normalize, float* d_out,
                                            void* stream, sred_run_info* info) {
  return sred_global_map_2d_shard_finish(c, d_sums, normalize, d_out, stream, info);
}

sred_status sred_global_map_2d_device(sred_ctx* c, const char* metric, const float* d_img, int w, int h, int bw,
                                      int bh, float relc, int normalize, float* d_out, void* stream,
                                      sred_run_info* info) {
  if (!c || !d_img || !d_out) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return global_core(c, m, d_img, w, h, bw, bh, relc, normalize, d_out, pick(c, stream), info, nullptr);
}

sred_status sred_calculate_block_repetition_map_2d(sred_ctx* c, const char* metric, const float* img, int w,
                                                   int h, const float* ref_pixels, int block_size, int bw, int bh,
                                                   float ref_mean, float ref_std, float relc, int normalize,
                                                   float* out) {
  if (!c || !img || !ref_pixels || !out) return SRED_ERR_ARG;
  const int m = block_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown block metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (w <= 0 || h <= 0) return fail(c, SRED_ERR_ARG, "bad dimensions");
  const size_t n = (size_t)w * h;
  float *d_img, *d_out;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_OUT, n, &d_out));
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CKS(block_core(c, m, d_img, w, h, 1, ref_pixels, block_size, bw, bh, ref_mean, ref_std, relc, normalize, d_out,
                 c->stream));
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_block_map_2d_stack(sred_ctx* c, const char* metric, const float* img, int w, int h, int frames,
                                    const float* ref_pixels, int block_size, int bw, int bh, float ref_mean,
                                    float ref_std, float relc, int normalize, int chunk_frames, float* out) {
  if (!c || !img || !ref_pixels || !out) return SRED_ERR_ARG;
  const int m = block_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown block metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (w <= 0 || h <= 0) return fail(c, SRED_ERR_ARG, "bad dimensions");
  if (frames < 1 || chunk_frames < 0) return fail(c, SRED_ERR_ARG, "frames must be >= 1 and chunk_frames >= 0");
  const size_t plane = (size_t)w * h;
  // default chunk: about 32 MiB of frames, so a chunk's copy is long enough
  // to hide the kernels of the neighbouring chunks and short enough to start
  // the pipeline quickly
  size_t chunk = chunk_frames > 0 ? (size_t)chunk_frames : ((size_t)32 << 20) / (plane * sizeof(float));
  chunk = std::max<size_t>(1, std::min<size_t>(chunk, std::min(frames, 65535)));
  const int nchunks = (int)((frames + chunk - 1) / chunk);
  const size_t slot = chunk * plane;
  float *d_in, *d_out;
  CKS(ensure(c, B_STKIN, 2 * slot, &d_in));
  CKS(ensure(c, B_STKOUT, 2 * slot, &d_out));
  if (!c->copy_in) CK(cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
  if (!c->copy_out) CK(cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking));
  // events: [0] start, then per slot s: in_ready, computed, out_done
  cudaEvent_t ev[7] = {};
  for (auto& e : ev) {
    const cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (r != cudaSuccess) {
      for (auto& x : ev)
        if (x) cudaEventDestroy(x);
      return cuda_fail(c, r, "sred_block_map_2d_stack: events");
    }
  }
  cudaEvent_t *in_ready = ev + 1, *computed = ev + 3, *out_done = ev + 5;
  auto drain = [&](sred_status st) {
    // no copy may still read or write the caller's buffers when this returns
    cudaStreamSynchronize(c->copy_in);
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->copy_out);
    for (auto& x : ev) cudaEventDestroy(x);
    if (st != SRED_OK) cudaGetLastError();
    return st;
  };
  // the slots may still be in use by earlier work on the context's stream
  {
    cudaError_t e = cudaEventRecord(ev[0], c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_in, ev[0], 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_out, ev[0], 0);
    if (e != cudaSuccess) return drain(cuda_fail(c, e, "sred_block_map_2d_stack"));
  }
  // Chunk i uses slot i % 2: its upload waits until the map of chunk i - 2
  // has read the slot, its map until its upload has landed and the download
  // of chunk i - 2 has left the output slot, its download until its map is
  // done. Uploads, maps and downloads of neighbouring chunks overlap.
  for (int i = 0; i < nchunks; i++) {
    const int s = i & 1;
    const size_t f0 = (size_t)i * chunk;
    const int nf = (int)std::min<size_t>(chunk, frames - f0);
    float* di = d_in + s * slot;
    float* dout = d_out + s * slot;
    cudaError_t e = cudaSuccess;
    if (i >= 2) e = cudaStreamWaitEvent(c->copy_in, computed[s], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(di, img + f0 * plane, nf * plane * sizeof(float), cudaMemcpyHostToDevice, c->copy_in);
    if (e == cudaSuccess) e = cudaEventRecord(in_ready[s], c->copy_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, in_ready[s], 0);
    if (e == cudaSuccess && i >= 2) e = cudaStreamWaitEvent(c->stream, out_done[s], 0);
    if (e != cudaSuccess) return drain(cuda_fail(c, e, "sred_block_map_2d_stack: upload"));
    sred_status st = block_core(c, m, di, w, h, nf, ref_pixels, block_size, bw, bh, ref_mean, ref_std, relc,
                                normalize, dout, c->stream);
    if (st != SRED_OK) return drain(st);
    e = cudaEventRecord(computed[s], c->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->copy_out, computed[s], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out + f0 * plane, dout, nf * plane * sizeof(float), cudaMemcpyDeviceToHost, c->copy_out);
    if (e == cudaSuccess) e = cudaEventRecord(out_done[s], c->copy_out);
    if (e != cudaSuccess) return drain(cuda_fail(c, e, "sred_block_map_2d_stack: download"));
  }
  cudaError_t e = cudaStreamSynchronize(c->copy_out);
  if (e != cudaSuccess) return drain(cuda_fail(c, e, "sred_block_map_2d_stack"));
  return drain(SRED_OK);
}

sred_status sred_block_map_2d_device(sred_ctx* c, const char* metric, const float* d_img, int w, int h,
                                     int frames, const float* ref_pixels, int block_size, int bw, int bh,
                                     float ref_mean, float ref_std, float relc, int normalize, float* d_out,
                                     void* stream) {
  if (!c || !d_img || !ref_pixels || !d_out) return SRED_ERR_ARG;
  const int m = block_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown block metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  const cudaStream_t st = pick(c, stream);
  CKS(block_core(c, m, d_img, w, h, frames, ref_pixels, block_size, bw, bh, ref_mean, ref_std, relc, normalize,
                 d_out, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

sred_status sred_set_gram_tuning(sred_ctx* c, int on) {
  if (!c) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->tune = on != 0;
  return SRED_OK;
}

int sred_gram_tuning_entries(int* entries, float* ms, int cap) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  int n = 0;
  for (const auto& kv : g_tune) {
    if (entries && ms && n < cap) {
      int* e = entries + 6 * n;
      e[0] = kv.first.kq;
      e[1] = kv.first.metric;
      e[2] = kv.first.nclass;
      e[3] = kv.second.choice.bn;
      e[4] = kv.second.choice.tr;
      e[5] = kv.second.choice.L;
      ms[n] = kv.second.ms;
    }
    n++;
  }
  return n;
}

sred_status sred_gram_tuning_set(int kq, int metric, int size_class, int bn, int tr, int max_l, float ms) {
  TcPlan p;
  TcChoice cand[16];
  const int nc = gram_tc_candidates(kq, cand, 16);
  bool ok = false;
  for (int i = 0; i < nc; i++) ok |= cand[i].bn == bn && cand[i].tr == tr && cand[i].L == max_l;
  if (!ok || size_class < 0 || size_class > 2 || !plan_gram_tc(kq, &p)) return SRED_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[TuneKey{kq, metric, size_class}] = TuneEntry{TcChoice{bn, tr, max_l}, ms};
  return SRED_OK;
}

sred_status sred_gram_tuning_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  return SRED_OK;
}

sred_status sred_debug_set_tc_wait(sred_ctx* c, unsigned long long timeout_ns, long long withhold_tile) {
  if (!c || withhold_tile < -1) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->tc_debug.timeout_ns = timeout_ns;
  c->tc_debug.withhold_tile = withhold_tile;
  return SRED_OK;
}

sred_status sred_debug_gram_rowdot(sred_ctx* c, int engine, const float* u, const float* w1, const float* w2, int n,
                                   int k, double* num, double* den) {
  if (!c || !u || !w1 || !w2 || !num || !den || n <= 0 || k <= 0 || k > kMaxK) return SRED_ERR_ARG;
  if (engine != SRED_ENGINE_TC && engine != SRED_ENGINE_FP32) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->shard.valid = false;  // overwrites workspaces of a prepared shard
  cudaSetDevice(c->device);
  cudaStream_t st = c->stream;
  const size_t n_pad = round_up((size_t)n, 256);
  const int kp = (int)round_up(k, 4), kq = (int)round_up(3 * k, 32);
  float *d_u, *d_U = nullptr, *d_rmax;
  __nv_bfloat16 *d_A = nullptr, *d_B = nullptr;
  BlockParams* d_params;
  double *d_num, *d_den;
  CKS(ensure(c, B_IMG, (size_t)n * k, &d_u));
  CKS(ensure(c, B_PARAMS, n_pad, &d_params));
  CKS(ensure(c, B_RMAX, n_pad / 128, &d_rmax));
  CKS(ensure(c, B_NUM, n_pad, &d_num));
  CKS(ensure(c, B_DEN, n_pad, &d_den));
  if (engine == SRED_ENGINE_FP32) {
    CKS(ensure(c, B_U, n_pad * kp, &d_U));
    CK(cudaMemsetAsync(d_U, 0, n_pad * kp * sizeof(float), st));
  } else {
    CKS(ensure(c, B_A, n_pad * kq, &d_A));
    CKS(ensure(c, B_B, n_pad * kq, &d_B));
    CK(cudaMemsetAsync(d_A, 0, n_pad * kq * sizeof(__nv_bfloat16), st));
    CK(cudaMemsetAsync(d_B, 0, n_pad * kq * sizeof(__nv_bfloat16), st));
  }
  std::vector<BlockParams> hp(n_pad);
  std::memset(hp.data(), 0, n_pad * sizeof(BlockParams));
  for (int i = 0; i < n; i++) { hp[i].a = w1[i]; hp[i].r = w2[i]; }
  CK(cudaMemcpyAsync(d_u, u, (size_t)n * k * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_params, hp.data(), n_pad * sizeof(BlockParams), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(d_rmax, 0, (n_pad / 128) * sizeof(float), st));
  CK(cudaMemsetAsync(d_num, 0, n_pad * sizeof(double), st));
  CK(cudaMemsetAsync(d_den, 0, n_pad * sizeof(double), st));
  k_pack_vectors<<<grid_for((size_t)n * 32, 256, 8 * c->num_sms), 256, 0, st>>>(
      d_u, n, k, engine == SRED_ENGINE_FP32 ? 0 : 1, d_U, kp, d_A, d_B, kq);
  CK(cudaGetLastError());
  EpiConsts ec{kDebugDot, n, 1.0f, kC1, kC2};
  if (engine == SRED_ENGINE_FP32) {
    CK(launch_gram_fp32(d_U, kp, d_params, d_rmax, ec, d_num, d_den, c->num_sms, st));
  } else {
    int* d_status;
    CKS(ensure(c, B_STATUS, 4, &d_status));
    CK(cudaMemsetAsync(d_status, 0, 4 * sizeof(int), st));
    float* d_soa;
    CKS(ensure(c, B_COLSOA, gram_tc_soa_floats((int)n_pad), &d_soa));
    TcPlan plan;
    if (!plan_gram_tc(kq, &plan)) return fail(c, SRED_ERR_ARG, "K too large for the tensor-core engine");
    CK(launch_gram_tc(d_A, d_B, kq, (int)n_pad, d_params, d_soa, ec, d_num, d_den, c->num_sms, d_status, st, 0, 1,
                      &c->tc_debug));
    int status = 0;
    CK(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (status) return fail(c, SRED_ERR_TIMEOUT, "tensor-core pipeline wait exceeded its bound");
  }
  CK(cudaMemcpyAsync(num, d_num, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(den, d_den, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// Shape metrics on host memory: the reference's Hu and phase-correlation
// kernels (shipped in src/main/resources/, never loaded by its Java code).
// ---------------------------------------------------------------------------

namespace {

// Interior extent of the all-pairs shape maps.
sred_status shape_interior(sred_ctx* c, int w, int h, const Ellipse& e, int* nx, int* ny) {
  *nx = w - 2 * e.rw;
  *ny = h - 2 * e.rh;
  if (*nx <= 0 || *ny <= 0) return fail(c, SRED_ERR_ARG, "image has no interior block");
  return SRED_OK;
}

// Uploads img, local means and stds; zeroes the output map.
sred_status shape_inputs(sred_ctx* c, const float* img, const float* means, const float* stds, size_t n,
                         float** d_img, float** d_m, float** d_s, float** d_out) {
  cudaStream_t st = c->stream;
  CKS(ensure(c, B_IMG, n, d_img));
  CKS(ensure(c, B_MEANS, n, d_m));
  CKS(ensure(c, B_STDS, n, d_s));
  CKS(ensure(c, B_OUT, n, d_out));
  CK(cudaMemcpyAsync(*d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(*d_m, means, n * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(*d_s, stds, n * sizeof(float), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(*d_out, 0, n * sizeof(float), st));
  return SRED_OK;
}

}  // namespace

sred_status sred_patch_hu_map_2d(sred_ctx* c, const float* patch, const float* img, int w, int h, int bw, int bh,
                                 int patch_size, float* out) {
  if (!c || !patch || !img || !out || patch_size <= 0) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  Ellipse e;
  CKS(check_block(c, w, h, bw, bh, &e));
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  const size_t n = (size_t)w * h;
  cudaStream_t st = c->stream;
  float *d_img, *d_out;
  CKS(ensure(c, B_IMG, n, &d_img));
  CKS(ensure(c, B_OUT, n, &d_out));
  CK(cudaMemcpyAsync(d_img, img, n * sizeof(float), cudaMemcpyHostToDevice, st));
  k_patch_hu<<<dim3((unsigned)((n + 127) / 128), 1), 128, 0, st>>>(d_img, w, h, e, patch_size,
                                                                    patch_hu1(patch, bw, bh), d_out, nullptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

sred_status sred_hu_map_2d(sred_ctx* c, const float* img, const float* local_means, const float* local_stds, int w,
                           int h, int bw, int bh, float* out) {
  if (!c || !img || !local_means || !local_stds || !out) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  Ellipse e;
  int nx, ny;
  CKS(check_block(c, w, h, bw, bh, &e));
  CKS(shape_interior(c, w, h, e, &nx, &ny));
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  const size_t n = (size_t)w * h;
  const int ni = nx * ny;
  cudaStream_t st = c->stream;
  float *d_img, *d_m, *d_s, *d_out, *d_feat, *d_sig;
  CKS(shape_inputs(c, img, local_means, local_stds, n, &d_img, &d_m, &d_s, &d_out));
  CKS(ensure(c, B_FEAT, ni, &d_feat));
  CKS(ensure(c, B_SIG, ni, &d_sig));
  k_hu_features<<<(ni + 127) / 128, 128, 0, st>>>(d_img, d_m, d_s, w, bw, bh, nx, ni, d_feat, d_sig);
  k_hu_pairs<<<(ni + 255) / 256, 256, 0, st>>>(d_feat, d_sig, ni, w, e.rw, e.rh, nx, d_out);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

sred_status sred_phase_correlation_map_2d(sred_ctx* c, const float* img, const float* local_means,
                                          const float* local_stds, int w, int h, int bw, int bh, float* out) {
  if (!c || !img || !local_means || !local_stds || !out) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  Ellipse e;
  int nx, ny;
  CKS(check_block(c, w, h, bw, bh, &e));
  if (bw > kPhaseMaxDim || bh > kPhaseMaxDim)
    return fail(c, SRED_ERR_ARG, "phase correlation supports blocks up to 15x15");
  CKS(shape_interior(c, w, h, e, &nx, &ny));
  if (fault("launch")) return fail(c, SRED_ERR_LAUNCH, "injected launch failure");
  const size_t n = (size_t)w * h;
  const int ni = nx * ny, nn = bw * bh;
  cudaStream_t st = c->stream;
  float *d_img, *d_m, *d_s, *d_out, *d_sig;
  double *d_fr, *d_fi;
  CKS(shape_inputs(c, img, local_means, local_stds, n, &d_img, &d_m, &d_s, &d_out));
  CKS(ensure(c, B_SIG, ni, &d_sig));
  CKS(ensure(c, B_FR, (size_t)ni * nn, &d_fr));
  CKS(ensure(c, B_FI, (size_t)ni * nn, &d_fi));
  k_phase_dft<<<(ni + 127) / 128, 128, 0, st>>>(d_img, d_m, d_s, w, bw, bh, nx, ni, d_fr, d_fi);
  k_gather_interior<<<(ni + 255) / 256, 256, 0, st>>>(d_s, w, e.rw, e.rh, nx, ni, d_sig);
  launch_phase_pairs(d_fr, d_fi, d_sig, ni, bw, bh, w, nx, d_out, st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// Variance stabilisation (generalised Anscombe transform)
// ---------------------------------------------------------------------------

namespace {

// The objective of GATMinimizer2D for one parameter set, the image already on
// the device.
// Runs per block of the objective's moments kernels: enough CTAs for about
// four per SM, each run at least 1,024 elements, at most 64 runs.
int gat_runs(const sred_ctx* c, size_t nb, size_t per_block) {
  size_t r = (4 * (size_t)c->num_sms + nb - 1) / std::max<size_t>(nb, 1);
  r = std::min<size_t>(r, std::max<size_t>(1, per_block / 1024));
  return (int)std::max<size_t>(1, std::min<size_t>(r, 64));
}

// The per-block [sum, sum of squares] of each of np points from the runs'
// partial sums, added in run order in FP64 on the host.
sred_status gat_block_sums(sred_ctx* c, const double* d_part, int np, size_t nb, int runs,
                           std::vector<double>* sums) {
  std::vector<double> part(2 * (size_t)np * nb * runs);
  CK(cudaMemcpyAsync(part.data(), d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  sums->assign(2 * (size_t)np * nb, 0.0);
  for (size_t pb = 0; pb < (size_t)np * nb; pb++)
    for (int s = 0; s < runs; s++) {
      (*sums)[2 * pb] += part[2 * (pb * runs + s)];
      (*sums)[2 * pb + 1] += part[2 * (pb * runs + s) + 1];
    }
  return SRED_OK;
}

// GATMinimizer2D.userFunction at np <= kGatMaxPoints points p[i] = (gain,
// sigma, offset), one launch for all of them.
sred_status gat_objective_dev(sred_ctx* c, const float* d_img, int w, int h, const double (*p)[3], int np,
                              double* error) {
  int bw, bh, nbx, nby;
  if (!gat_grid(w, h, &bw, &bh, &nbx, &nby)) return fail(c, SRED_ERR_ARG, "image too small for the GAT fit (width and height >= 12)");
  const int nb = nbx * nby;
  const int runs = gat_runs(c, (size_t)nb, (size_t)bw * bh);
  double* d_sums;
  CKS(ensure(c, B_GAT, 2 * (size_t)kGatMaxPoints * nb * runs, &d_sums));
  GatPoints pts;
  for (int i = 0; i < np; i++) {
    pts.gain[i] = p[i][0];
    pts.c[i] = (3.0 / 8.0) * p[i][0] * p[i][0] + p[i][1] * p[i][1] - p[i][0] * p[i][2];
  }
  k_gat_block_moments<<<dim3(nb, runs, np), 256, 0, c->stream>>>(d_img, w, bw, bh, nbx, pts, d_sums);
  CK(cudaGetLastError());
  std::vector<double> sums;
  CKS(gat_block_sums(c, d_sums, np, (size_t)nb, runs, &sums));
  for (int i = 0; i < np; i++) error[i] = gat_error(sums.data() + 2 * (size_t)i * nb, nb, bw, bh);
  return SRED_OK;
}

// GATMinimizer3D.userFunction (java/GATMinimizer3D.java): NaN outside gain > 0,
// sigma >= 0, offset >= 0; block grid of width/6 x height/6 x depth/6 voxels
// (at least 1), halved along every axis with fewer than 2 blocks until each
// has 2 or the block is one voxel; per-block variance with FP64 sums of the
// transformed voxels (as float, then widened). np <= kGatMaxPoints points,
// the ones inside the domain in one launch.
sred_status gat_objective3d_dev(sred_ctx* c, const float* d_vol, int w, int h, int d, const double (*p)[3], int np,
                                double* error) {
  int in[kGatMaxPoints], nin = 0;
  for (int i = 0; i < np; i++) {
    if (p[i][0] <= 0 || p[i][1] < 0 || p[i][2] < 0)
      error[i] = std::nan("");
    else
      in[nin++] = i;
  }
  if (nin == 0) return SRED_OK;
  int bw, bh, bd, nbx, nby, nbz;
  gat3d_grid(w, h, d, &bw, &bh, &bd, &nbx, &nby, &nbz);
  const size_t nb = (size_t)nbx * nby * nbz;
  if (nb == 0) return fail(c, SRED_ERR_ARG, "volume too small for the GAT fit");
  const int runs = gat_runs(c, nb, (size_t)bw * bh * bd);
  double* d_sums;
  CKS(ensure(c, B_GAT, 2 * (size_t)kGatMaxPoints * nb * runs, &d_sums));
  GatPoints pts;
  for (int k = 0; k < nin; k++) {
    const double* q = p[in[k]];
    pts.gain[k] = q[0];
    pts.c[k] = (3.0 / 8.0) * q[0] * q[0] + q[1] * q[1] - q[0] * q[2];
  }
  k_gat_block_moments3d<<<dim3((unsigned)nb, runs, nin), 256, 0, c->stream>>>(d_vol, w, h, bw, bh, bd, nbx, nby,
                                                                               pts, d_sums);
  CK(cudaGetLastError());
  std::vector<double> sums;
  CKS(gat_block_sums(c, d_sums, nin, nb, runs, &sums));
  for (int k = 0; k < nin; k++) error[in[k]] = gat_error(sums.data() + 2 * (size_t)k * nb, (int)nb, bw * bh * bd, 1);
  return SRED_OK;
}

}  // namespace

sred_status sred_gat_2d(sred_ctx* c, float* img, int w, int h, double gain, double sigma, double offset) {
  if (!c || !img || w <= 0 || h <= 0 || !(gain != 0.0)) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h;
  float* d;
  CKS(ensure(c, B_IMG, n, &d));
  CK(cudaMemcpyAsync(d, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  const double cst = (3.0 / 8.0) * gain * gain + sigma * sigma - gain * offset;
  k_gat<<<grid_for(n, 256, 8 * c->num_sms), 256, 0, c->stream>>>(d, n, gain, cst);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(img, d, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_gat_objective_2d(sred_ctx* c, const float* img, int w, int h, double gain, double sigma,
                                  double offset, double* error) {
  if (!c || !img || !error || w <= 0 || h <= 0) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h;
  float* d;
  CKS(ensure(c, B_IMG, n, &d));
  CK(cudaMemcpyAsync(d, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  const double p[1][3] = {{gain, sigma, offset}};
  return gat_objective_dev(c, d, w, h, p, 1, error);
}

// Nelder-Mead downhill simplex (Nelder & Mead, Computer Journal 7:308, 1965;
// reflection 1, expansion 2, contraction 1/2, shrink 1/2) over (gain, sigma,
// offset) from x0 with the initial steps of the reference's Minimizer set-up
// (1, 10, 100; java/GATMinimizer2D.java:42-45). An objective of NaN ranks
// last. Stops after max_iter evaluations or when the simplex's objective
// values agree to 1e-15 of the best.
// objective(p, np, out) evaluates np <= 4 points in one go. Each iteration
// evaluates the reflection, the expansion and both contractions together and
// then takes the same decisions as evaluating them one at a time, so the
// simplex path is the sequential one; `evals` counts only the evaluations
// the sequential method makes.
extern "C++" {
template <class F>
sred_status nelder_mead3(F objective, int max_iter, double* x0, double* f_best) {
  double x[4][3];
  double f[4];
  const double step[3] = {1.0, 10.0, 100.0};
  auto batch = [&](const double (*p)[3], int np, double* out) -> sred_status {
    const sred_status st = objective(p, np, out);
    if (st != SRED_OK) return st;
    for (int i = 0; i < np; i++)
      if (std::isnan(out[i])) out[i] = HUGE_VAL;
    return SRED_OK;
  };
  for (int v = 0; v < 4; v++) {
    for (int k = 0; k < 3; k++) x[v][k] = x0[k];
    if (v > 0) x[v][v - 1] += step[v - 1];
  }
  sred_status st = batch(x, 4, f);
  if (st != SRED_OK) return st;
  int evals = 4;
  while (evals < max_iter) {
    int order[4] = {0, 1, 2, 3};
    std::sort(order, order + 4, [&](int a, int b) { return f[a] < f[b]; });
    const int best = order[0], worst = order[3], second = order[2];
    if (std::fabs(f[worst] - f[best]) <= 1e-15 * std::fabs(f[best])) break;
    double cen[3] = {0, 0, 0};
    for (int v = 0; v < 4; v++)
      if (v != worst)
        for (int k = 0; k < 3; k++) cen[k] += x[v][k] / 3.0;
    // candidates: reflection, expansion, outside and inside contraction
    double cand[4][3], fc4[4];
    for (int k = 0; k < 3; k++) {
      cand[0][k] = cen[k] + (cen[k] - x[worst][k]);
      cand[1][k] = cen[k] + 2.0 * (cen[k] - x[worst][k]);
      cand[2][k] = cen[k] + 0.5 * (cand[0][k] - cen[k]);
      cand[3][k] = cen[k] + 0.5 * (x[worst][k] - cen[k]);
    }
    st = batch(cand, 4, fc4);
    if (st != SRED_OK) return st;
    const double fr = fc4[0];
    evals++;
    if (fr < f[best]) {
      const double fe = fc4[1];
      evals++;
      const int pick = fe < fr ? 1 : 0;
      std::copy(cand[pick], cand[pick] + 3, x[worst]);
      f[worst] = fc4[pick];
    } else if (fr < f[second]) {
      std::copy(cand[0], cand[0] + 3, x[worst]);
      f[worst] = fr;
    } else {
      const bool outside = fr < f[worst];
      const int ic = outside ? 2 : 3;
      const double fc = fc4[ic];
      evals++;
      if (fc < (outside ? fr : f[worst])) {
        std::copy(cand[ic], cand[ic] + 3, x[worst]);
        f[worst] = fc;
      } else {
        double sx[3][3], sf[3];
        int idx[3], ns = 0;
        for (int v = 0; v < 4; v++)
          if (v != best) {
            for (int k = 0; k < 3; k++) sx[ns][k] = x[best][k] + 0.5 * (x[v][k] - x[best][k]);
            idx[ns++] = v;
          }
        st = batch(sx, 3, sf);
        if (st != SRED_OK) return st;
        for (int q = 0; q < 3; q++) {
          std::copy(sx[q], sx[q] + 3, x[idx[q]]);
          f[idx[q]] = sf[q];
        }
        evals += 3;
      }
    }
  }
  int best = 0;
  for (int v = 1; v < 4; v++)
    if (f[v] < f[best]) best = v;
  for (int k = 0; k < 3; k++) x0[k] = x[best][k];
  *f_best = f[best];
  return SRED_OK;
}
}  // extern "C++"

// The GAT parameters minimising the objective of java/GATMinimizer2D.java, with
// the image resident.
sred_status sred_gat_fit_2d(sred_ctx* c, const float* img, int w, int h, int max_iter, double* gain, double* sigma,
                            double* offset, double* error_out) {
  if (!c || !img || !gain || !sigma || !offset || w <= 0 || h <= 0 || max_iter < 1) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h;
  float* d;
  CKS(ensure(c, B_IMG, n, &d));
  CK(cudaMemcpyAsync(d, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  double x[3] = {*gain, *sigma, *offset}, fb;
  CKS(nelder_mead3([&](const double (*p)[3], int np, double* out) { return gat_objective_dev(c, d, w, h, p, np, out); },
                   max_iter, x, &fb));
  *gain = x[0];
  *sigma = x[1];
  *offset = x[2];
  if (error_out) *error_out = fb;
  return SRED_OK;
}

// ---- 3D (java/GATMinimizer3D.java) ----

sred_status sred_gat_3d(sred_ctx* c, float* vol, int w, int h, int d, double gain, double sigma, double offset) {
  if (!c || !vol || w <= 0 || h <= 0 || d <= 0) return SRED_ERR_ARG;
  return sred_gat_2d(c, vol, w, h * d, gain, sigma, offset);
}

sred_status sred_gat_objective_3d(sred_ctx* c, const float* vol, int w, int h, int d, double gain, double sigma,
                                  double offset, double* error) {
  if (!c || !vol || !error || w <= 0 || h <= 0 || d <= 0) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h * d;
  float* dv;
  CKS(ensure(c, B_IMG, n, &dv));
  CK(cudaMemcpyAsync(dv, vol, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  const double p[1][3] = {{gain, sigma, offset}};
  return gat_objective3d_dev(c, dv, w, h, d, p, 1, error);
}

sred_status sred_gat_fit_3d(sred_ctx* c, const float* vol, int w, int h, int d, int max_iter, double* gain,
                            double* sigma, double* offset, double* error_out) {
  if (!c || !vol || !gain || !sigma || !offset || w <= 0 || h <= 0 || d <= 0 || max_iter < 1) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h * d;
  float* dv;
  CKS(ensure(c, B_IMG, n, &dv));
  CK(cudaMemcpyAsync(dv, vol, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  double x[3] = {*gain, *sigma, *offset}, fb;
  CKS(nelder_mead3(
      [&](const double (*p)[3], int np, double* out) { return gat_objective3d_dev(c, dv, w, h, d, p, np, out); },
      max_iter, x, &fb));
  *gain = x[0];
  *sigma = x[1];
  *offset = x[2];
  if (error_out) *error_out = fb;
  return SRED_OK;
}

// java/Utils.java:557-639 on host memory (ImageJ's float conversion is the caller's).
sred_status sred_reference_block_2d(const float* blk, int bw, int bh, float* pixels, int* block_size, float* mean,
                                    float* std_out) {
  if (!blk || !pixels || !block_size || !mean || !std_out) return SRED_ERR_ARG;
  if (bw % 2 == 0 || bh % 2 == 0 || bw < 3 || bh < 3) return SRED_ERR_ARG;
  Ellipse e;
  const int K = build_ellipse(bw, bh, &e);
  if (K < 2 || K > kMaxK) return SRED_ERR_ARG;
  for (int i = 0; i < K; i++) pixels[i] = blk[(e.dy[i] + e.rh) * bw + (e.dx[i] + e.rw)];
  float mn = 3.40282347e38f, mx = -3.40282347e38f;
  for (int i = 0; i < K; i++) {
    mn = std::min(mn, pixels[i]);
    mx = std::max(mx, pixels[i]);
  }
  float m = 0.0f;
  for (int i = 0; i < K; i++) {
    pixels[i] = (pixels[i] - mn) / (mx - mn + kEps);
    m += pixels[i];
  }
  m /= (float)K;
  for (int i = 0; i < K; i++) pixels[i] = pixels[i] - m;
  float sd = 0.0f;
  for (int i = 0; i < K; i++) sd += (pixels[i] - m) * (pixels[i] - m);
  sd = (float)std::sqrt((double)(sd / ((float)(K - 1))));
  *block_size = K;
  *mean = m;
  *std_out = sd;
  return SRED_OK;
}

sred_status sred_normalize_image_2d(float* a, int w, int h, int bw_, int bh_, const float* mask) {
  if (!a || w <= 0 || h <= 0) return SRED_ERR_ARG;
  float mn = 3.40282347e38f, mx = -3.40282347e38f;
  for (int y = bh_; y < h - bh_; y++)
    for (int x = bw_; x < w - bw_; x++) {
      const int i = y * w + x;
      if (mask) {
        if (mask[i] != 0.0f && mask[i] != 1.0f) return SRED_ERR_ARG;
        if (!(mask[i] > 0.0f)) continue;
      }
      mn = std::min(a[i], mn);
      mx = std::max(a[i], mx);
    }
  for (int y = bh_; y < h - bh_; y++)
    for (int x = bw_; x < w - bw_; x++) {
      const int i = y * w + x;
      if (mask && !(mask[i] > 0.0f)) continue;
      a[i] = (a[i] - mn) / (mx - mn + kEps);
    }
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// 3D block repetition maps
// ---------------------------------------------------------------------------

int sred_block_size_3d(int bw, int bh, int bd) {
  if (bw < 3 || bh < 3 || bd < 3) return 0;
  return build_ellipsoid(bw, bh, bd, 1, 1, nullptr);
}

sred_status sred_reference_block_3d(const float* blk, int bw, int bh, int bd, float* pixels, int* block_size,
                                    float* mean, float* std_out) {
  if (!blk || !pixels || !block_size || !mean || !std_out) return SRED_ERR_ARG;
  if (bw % 2 == 0 || bh % 2 == 0 || bd % 2 == 0 || bw < 3 || bh < 3 || bd < 3) return SRED_ERR_ARG;
  const int rw = bw / 2, rh = bh / 2, rd = bd / 2;
  const int K = build_ellipsoid(bw, bh, bd, 1, 1, nullptr);
  if (K < 2 || K > kMaxK3) return SRED_ERR_ARG;
  int k = 0;
  for (int z = 0; z < bd; z++)
    for (int y = 0; y < bh; y++)
      for (int x = 0; x < bw; x++) {
        const float fx = (float)(x - rw), fy = (float)(y - rh), fz = (float)(z - rd);
        if (((fx * fx) / (float)(rw * rw)) + ((fy * fy) / (float)(rh * rh)) + ((fz * fz) / (float)(rd * rd)) <=
            1.0f)
          pixels[k++] = blk[((size_t)z * bh + y) * bw + x];
      }
  // normalizeArray, minus the mean, normalizeArray again (java/Utils.java:1100-1140)
  auto minmax = [&]() {
    float mn = 3.40282347e38f, mx = -3.40282347e38f;
    for (int i = 0; i < K; i++) {
      mn = std::min(pixels[i], mn);
      mx = std::max(pixels[i], mx);
    }
    for (int i = 0; i < K; i++) pixels[i] = (pixels[i] - mn) / (mx - mn + kEps);
  };
  auto mean_of = [&]() {
    float m = 0.0f;
    for (int i = 0; i < K; i++) m += pixels[i];
    return m / (float)K;
  };
  minmax();
  float m = mean_of();
  for (int i = 0; i < K; i++) pixels[i] = pixels[i] - m;
  minmax();
  m = mean_of();
  float sd = 0.0f;
  for (int i = 0; i < K; i++) sd += (pixels[i] - m) * (pixels[i] - m);
  *block_size = K;
  *mean = m;
  *std_out = (float)std::sqrt((double)(sd / ((float)(K - 1))));
  return SRED_OK;
}

sred_status sred_local_statistics_3d(sred_ctx* c, const float* vol, int w, int h, int d, int bw, int bh, int bd,
                                     float* means, float* stds) {
  if (!c || !vol || !means || !stds) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  cudaStream_t st = c->stream;
  Vol3 v;
  int* d_off;
  CKS(prepare_volume(c, w, h, d, bw, bh, bd, st, &v, &d_off));
  const size_t n = (size_t)w * h * d;
  float *d_vol, *d_m, *d_s;
  CKS(ensure(c, B_IMG, n, &d_vol));
  CKS(ensure(c, B_MEANS, n, &d_m));
  CKS(ensure(c, B_STDS, n, &d_s));
  CK(cudaMemcpyAsync(d_vol, vol, n * sizeof(float), cudaMemcpyHostToDevice, st));
  k_local_stats3d<<<vol_grid(v), dim3(32, 4), sizeof(int) * v.k, st>>>(d_vol, v, d_off, d_m, d_s);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(means, d_m, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(stds, d_s, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

sred_status sred_relevance_mask_3d(sred_ctx* c, int w, int h, int d, int bw, int bh, int bd, const float* stds,
                                   float relc, float* mask, float* noise_var) {
  if (!c || !stds || !mask || !noise_var) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  cudaStream_t st = c->stream;
  Vol3 v;
  int* d_off;
  CKS(prepare_volume(c, w, h, d, bw, bh, bd, st, &v, &d_off));
  const size_t n = (size_t)w * h * d;
  float *d_s, *d_m;
  CKS(ensure(c, B_STDS, n, &d_s));
  CKS(ensure(c, B_MASK, n, &d_m));
  CK(cudaMemcpyAsync(d_s, stds, n * sizeof(float), cudaMemcpyHostToDevice, st));
  CKS(mask_3d(c, v, d_s, relc, d_m, nullptr, st, noise_var));
  CK(cudaMemcpyAsync(mask, d_m, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return SRED_OK;
}

sred_status sred_calculate_block_repetition_map_3d(sred_ctx* c, const char* metric, const float* vol, int w,
                                                   int h, int d, const float* ref_pixels, int block_size, int bw,
                                                   int bh, int bd, float ref_mean, float ref_std, float relc,
                                                   int normalize, float* out) {
  if (!c || !vol || !ref_pixels || !out) return SRED_ERR_ARG;
  const int m = block_metric(metric);
  if (m < kPearson || m > kAbsDiff) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown 3D block metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (w <= 0 || h <= 0 || d <= 0) return fail(c, SRED_ERR_ARG, "bad dimensions");
  const size_t n = (size_t)w * h * d;
  float *d_vol, *d_out;
  CKS(ensure(c, B_IMG, n, &d_vol));
  CKS(ensure(c, B_OUT, n, &d_out));
  CKS(block3d_core(c, m, d_vol, w, h, d, ref_pixels, block_size, bw, bh, bd, ref_mean, ref_std, relc, normalize,
                   d_out, c->stream, vol));
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_block_map_3d_device(sred_ctx* c, const char* metric, const float* d_vol, int w, int h, int d,
                                     const float* ref_pixels, int block_size, int bw, int bh, int bd, float ref_mean,
                                     float ref_std, float relc, int normalize, float* d_out, void* stream) {
  if (!c || !d_vol || !ref_pixels || !d_out) return SRED_ERR_ARG;
  const int m = block_metric(metric);
  if (m < kPearson || m > kAbsDiff) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown 3D block metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return block3d_core(c, m, d_vol, w, h, d, ref_pixels, block_size, bw, bh, bd, ref_mean, ref_std, relc, normalize,
                      d_out, pick(c, stream));
}

sred_status sred_calculate_global_repetition_map_3d(sred_ctx* c, const char* metric, const float* vol, int w,
                                                    int h, int d, int bw, int bh, int bd, float relc, int normalize,
                                                    float* out, sred_run_info* info) {
  if (!c || !vol || !out) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  if (w <= 0 || h <= 0 || d <= 0) return fail(c, SRED_ERR_ARG, "bad dimensions");
  const size_t n = (size_t)w * h * d;
  float *d_vol, *d_out;
  CKS(ensure(c, B_IMG, n, &d_vol));
  CKS(ensure(c, B_OUT, n, &d_out));
  CK(cudaMemcpyAsync(d_vol, vol, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CKS(global3d_core(c, m, d_vol, w, h, d, bw, bh, bd, relc, normalize, d_out, c->stream, info));
  CK(cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_global_map_3d_device(sred_ctx* c, const char* metric, const float* d_vol, int w, int h, int d,
                                      int bw, int bh, int bd, float relc, int normalize, float* d_out, void* stream,
                                      sred_run_info* info) {
  if (!c || !d_vol || !d_out) return SRED_ERR_ARG;
  const int m = global_metric(metric);
  if (m < 0) return fail(c, SRED_ERR_UNKNOWN_METRIC, "unknown global metric");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  return global3d_core(c, m, d_vol, w, h, d, bw, bh, bd, relc, normalize, d_out, pick(c, stream), info);
}

// ---------------------------------------------------------------------------
// Relevance-mask tools
// ---------------------------------------------------------------------------

sred_status sred_relevance_mask_tool_2d(sred_ctx* c, const float* img, int w, int h, int bw, int bh,
                                        float filter_constant, float* mask, float* threshold, float* noise_var) {
  if (!c || !img || !mask || !threshold || !noise_var) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  Ellipse e;
  float *d_img, *d_stat;
  CKS(tool_stat(c, img, w, h, bw, bh, 1, &e, &d_img, &d_stat));
  float nv;
  CKS(tool_noise_var(c, d_img, w, h, true, c->stream, &nv));
  const float thr = tool_threshold(nv, filter_constant);
  CKS(tool_masks(c, d_stat, w, h, e, &thr, 1, mask));
  *threshold = thr;
  *noise_var = nv;
  return SRED_OK;
}

sred_status sred_relevance_mask_sweep_2d(sred_ctx* c, const float* img, int w, int h, int bw, int bh, float lower,
                                         float step, int n, float* masks, float* constants, float* noise_var) {
  if (!c || !img || !masks || !constants || !noise_var) return SRED_ERR_ARG;
  if (n < 1 || n > 65535) return fail(c, SRED_ERR_ARG, "the number of masks must be in 1..65535");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  Ellipse e;
  float *d_img, *d_stat;
  CKS(tool_stat(c, img, w, h, bw, bh, 0, &e, &d_img, &d_stat));
  float nv;
  CKS(tool_noise_var(c, d_img, w, h, false, c->stream, &nv));
  std::vector<float> thr(n);
  float fc = lower;
  for (int i = 0; i < n; i++) {
    constants[i] = fc;
    thr[i] = tool_threshold(nv, fc);
    fc += step;
  }
  CKS(tool_masks(c, d_stat, w, h, e, thr.data(), n, masks));
  *noise_var = nv;
  return SRED_OK;
}

sred_status sred_relevance_constant_range_2d(sred_ctx* c, const float* img, int w, int h, int bw, int bh,
                                             float step, float* all_ones, float* all_zeros, float* noise_var) {
  if (!c || !img || !all_ones || !all_zeros || !noise_var) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  Ellipse e;
  float *d_img, *d_stat;
  CKS(tool_stat(c, img, w, h, bw, bh, 0, &e, &d_img, &d_stat));
  float nv;
  CKS(tool_noise_var(c, d_img, w, h, false, c->stream, &nv));
  unsigned* mm;
  CKS(ensure(c, B_MM, 2, &mm));
  const unsigned init[2] = {0xffffffffu, 0u};
  CK(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, c->stream));
  k_stat_sq_minmax<<<grid_for((size_t)w * h, 256, 4 * c->num_sms), 256, 0, c->stream>>>(d_stat, w, h, e.rw, e.rh,
                                                                                        mm);
  CK(cudaGetLastError());
  unsigned hm[2];
  CK(cudaMemcpyAsync(hm, mm, sizeof(hm), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // The reference's loop (OptimiseRelevanceMask_.run): c = 0, step, 2 step, ...
  // (FP32 accumulation) until the mask is all 0, remembering the last c whose
  // interior is all 1. One pixel is 1 at c iff !(s^2 < thr) and s^2 != 0, so
  // the interior's smallest and largest s^2 decide every step.
  const bool any = hm[0] != 0xffffffffu;
  float mn = 0.0f, mx = 0.0f;
  std::memcpy(&mn, &hm[0], sizeof(float));
  std::memcpy(&mx, &hm[1], sizeof(float));
  float fc = 0.0f, ones = 0.0f;
  for (;;) {
    const float thr = tool_threshold(nv, fc);
    if (!any || (!(mn < thr) && mn != 0.0f)) ones = fc;
    if (!any || mx < thr || mx == 0.0f) break;
    const float next = fc + step;
    if (!(next > fc))
      return fail(c, SRED_ERR_ARG, "the relevance constant step never reaches an all-zero mask");
    fc = next;
  }
  *all_ones = ones;
  *all_zeros = fc;
  *noise_var = nv;
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// Redundancy classification
// ---------------------------------------------------------------------------

sred_status sred_classify_redundancy_2d(sred_ctx* c, const float* map, int w, int h, int border, int k,
                                        int optimal_k, int max_k, int64_t seed, float* out, int* k_used,
                                        double* wcss_out) {
  if (!c || !map || !out) return SRED_ERR_ARG;
  if (border < 0 || w - 2 * border < 1 || h - 2 * border < 1) return fail(c, SRED_ERR_ARG, "border leaves no pixels");
  const int kk = optimal_k ? max_k : k;
  if (kk < 1 || kk > kKmMaxK) return fail(c, SRED_ERR_ARG, "number of classes must be in 1..64");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  cudaStream_t s = c->stream;
  KmState st;
  st.n = (size_t)(w - 2 * border) * (h - 2 * border);
  if (st.n > (size_t)INT32_MAX) return fail(c, SRED_ERR_ARG, "map too large");
  if ((size_t)kk > st.n) return fail(c, SRED_ERR_ARG, "more classes than pixels");
  st.nblk = (int)((st.n + kKmSpan - 1) / kKmSpan);
  float* d_map;
  CKS(ensure(c, B_IMG, (size_t)w * h, &d_map));
  CKS(ensure(c, B_KMX, st.n, &st.x));
  CKS(ensure(c, B_KMD2, st.n, &st.d2));
  CKS(ensure(c, B_KMLAB, st.n, &st.lab));
  CKS(ensure(c, B_NMASK, 1, &st.changed));
  CKS(ensure(c, B_VARS, 2 * (size_t)st.nblk, &st.blk));
  CK(cudaMemcpyAsync(d_map, map, sizeof(float) * w * h, cudaMemcpyHostToDevice, s));
  k_km_gather<<<grid_for(st.n, 256, 8 * c->num_sms), 256, 0, s>>>(d_map, w, h, border, st.x);
  CK(cudaGetLastError());
  JavaRandom rng(seed);
  std::vector<double> centers, counts;
  double wcss = 0.0;
  int k_final = k;
  if (optimal_k) {
    // elbow (ClassifyRedundancy_.getOptimalK): the first k whose WCSS does not
    // drop below the previous one ends the search at the previous k
    double prev = DBL_MAX;
    k_final = 1;
    for (int kt = 1; kt <= max_k; kt++) {
      CKS(kmeans_run(c, st, kt, rng, centers, counts, &wcss));
      if (wcss < prev) {
        prev = wcss;
        k_final = kt;
      } else {
        break;
      }
    }
  }
  CKS(kmeans_run(c, st, k_final, rng, centers, counts, &wcss));
  // ranks: clusters by point count, largest first, ties in cluster order
  const int kc = (int)centers.size();
  std::vector<int> order(kc), rank(kc);
  for (int j = 0; j < kc; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return counts[a] > counts[b]; });
  for (int j = 0; j < kc; j++) rank[order[j]] = j;
  int* d_rank;
  float* d_out;
  CKS(ensure(c, B_THR, kc, &d_rank));
  CKS(ensure(c, B_OUT, (size_t)w * h, &d_out));
  CK(cudaMemcpyAsync(d_rank, rank.data(), sizeof(int) * kc, cudaMemcpyHostToDevice, s));
  k_km_scatter<<<grid_for((size_t)w * h, 256, 8 * c->num_sms), 256, 0, s>>>(st.lab, d_rank, w, h, border, d_out);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_out, sizeof(float) * w * h, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (k_used) *k_used = kc;
  if (wcss_out) *wcss_out = wcss;
  return SRED_OK;
}

sred_status sred_debug_divide_fixed64(sred_ctx* c, const double* a, size_t n, double b, double* out) {
  if (!c || !a || !out) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  double *d_a, *d_o;
  CKS(ensure(c, B_IMG, n, &d_a));
  CKS(ensure(c, B_OUT, n, &d_o));
  CK(cudaMemcpyAsync(d_a, a, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  k_divide_fixed64<<<grid_for(n, 256, 8 * c->num_sms), 256, 0, c->stream>>>(d_a, n, b, d_o);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_o, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_debug_divide_fixed(sred_ctx* c, const float* a, size_t n, float b, float* out) {
  if (!c || !a || !out) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  float *d_a, *d_o;
  CKS(ensure(c, B_IMG, n, &d_a));
  CKS(ensure(c, B_OUT, n, &d_o));
  CK(cudaMemcpyAsync(d_a, a, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  k_divide_fixed<<<grid_for(n, 256, 8 * c->num_sms), 256, 0, c->stream>>>(d_a, n, b, d_o);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d_o, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

// ---------------------------------------------------------------------------
// Quadtree / octree variance stabilisation
// ---------------------------------------------------------------------------

sred_status sred_gat_quadtree_2d(sred_ctx* c, float* img, int w, int h, int min_size, float alpha, int max_iter,
                                 float lts_fraction, double* g0, double* edc, int* n_leaves) {
  if (!c || !img || !g0 || !edc || w <= 0 || h <= 0) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h;
  float* d;
  CKS(ensure(c, B_IMG, n, &d));
  CK(cudaMemcpyAsync(d, img, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CKS(gat_tree_core(c, d, w, h, 1, false, min_size, alpha, max_iter, lts_fraction, g0, edc, n_leaves));
  CK(cudaMemcpyAsync(img, d, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

sred_status sred_gat_octree_3d(sred_ctx* c, float* vol, int w, int h, int d, int min_size, float alpha, int max_iter,
                               float lts_fraction, double* g0, double* edc, int* n_leaves) {
  if (!c || !vol || !g0 || !edc || w <= 0 || h <= 0 || d <= 0) return SRED_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->shard.valid = false;
  const size_t n = (size_t)w * h * d;
  float* dv;
  CKS(ensure(c, B_IMG, n, &dv));
  CK(cudaMemcpyAsync(dv, vol, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CKS(gat_tree_core(c, dv, w, h, d, true, min_size, alpha, max_iter, lts_fraction, g0, edc, n_leaves));
  CK(cudaMemcpyAsync(vol, dv, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SRED_OK;
}

double sred_f_quantile(double p, double df) { return (p > 0.0 && p < 1.0 && df > 0.0) ? f_quantile_equal_df(p, df) : std::nan(""); }

}  // extern "C"
