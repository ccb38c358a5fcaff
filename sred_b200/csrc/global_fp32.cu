// Plain FP32 CUDA-core engine of the global repetition map.
//
// All-pairs Gram G = U U^T over the compacted relevant blocks (unit vectors,
// FP32), register-blocked 8x8 per thread on a 128x128 tile, with the fused
// per-pair epilogue (epilogue.cuh) reducing each row in registers: the N x N
// similarity matrix is never stored. Work items are (128-row block, range of
// 128-column tiles); a persistent grid walks them, so the triangular-free
// all-pairs work spreads evenly over the SMs. Row sums go to FP64 global
// accumulators with one atomic per row per item.
//
// This is the comparison form for the tensor-core engine: the same moments,
// compaction, work split and epilogue, with FFMA contraction. For NRMSE it
// accumulates |u_p - u_q|^2 instead (diff_metric), the form without
// cancellation for near-identical blocks; NRMSE always runs here.
#include <algorithm>

#include "common.cuh"
#include "epilogue.cuh"

namespace sred {

namespace {

constexpr int BM = 128;
constexpr int NT = 256;
constexpr int TM = 8;

struct Fp32Args {
  const float* U;
  int kp;
  const BlockParams* params;
  const float* tile_rmax;
  EpiConsts ec;
  double* num;
  double* den;
  int rb0;           // first 128-row block of this launch
  int n_rb;          // 128-row blocks of this launch
  int n_ct;          // 128-column tiles
  int ct_per_item;   // column tiles per work item
  int n_items;
};

// Load a 128 x kp tile (rows r0..r0+127 of U) into smem transposed: S[k][r].
__device__ __forceinline__ void load_tile_t(float* S, const float* __restrict__ U, int kp, int r0) {
  const int kp4 = kp >> 2;
  for (int i = threadIdx.x; i < BM * kp4; i += NT) {
    const int r = i / kp4, k4 = i - r * kp4;
    const float4 v = *reinterpret_cast<const float4*>(U + (size_t)(r0 + r) * kp + 4 * k4);
    S[(4 * k4 + 0) * (BM + 4) + r] = v.x;
    S[(4 * k4 + 1) * (BM + 4) + r] = v.y;
    S[(4 * k4 + 2) * (BM + 4) + r] = v.z;
    S[(4 * k4 + 3) * (BM + 4) + r] = v.w;
  }
}

template <int METRIC, int CMODE, bool FULL, bool DIAG>
__device__ __forceinline__ void tile_epilogue(const float (&acc)[TM][TM], const BlockParams* __restrict__ rowp,
                                              const BlockParams* __restrict__ colp, int row0, int col0,
                                              const EpiConsts& ec, float (&rn)[TM], float (&rd)[TM]) {
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
  for (int i = 0; i < TM; i++) {
    const RowState rs = make_row(rowp[ty * TM + i], ec);
    float sn = 0.0f, sd = 0.0f;
#pragma unroll
    for (int j = 0; j < TM; j++) {
      const int c = tx * TM + j;
      float G = acc[i][j];
      if (!diff_metric(METRIC) && DIAG && col0 + c == row0 + ty * TM + i && rs.r > 0.0f) G = 1.0f;
      if (FULL || col0 + c < ec.n) epi_pair<METRIC, CMODE>(G, rs, colp[c], ec, sn, sd);
    }
    rn[i] += sn;
    rd[i] += sd;
  }
}

template <int METRIC>
__global__ void __launch_bounds__(NT, 2) k_gram_fp32(Fp32Args g) {
  extern __shared__ __align__(16) float smem[];
  float* As = smem;                                  // [kp][BM+4]
  float* Bs = As + (size_t)g.kp * (BM + 4);          // [kp][BM+4]
  BlockParams* Ap = reinterpret_cast<BlockParams*>(Bs + (size_t)g.kp * (BM + 4));  // [BM]
  BlockParams* Bp = Ap + BM;                                                         // [BM]
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  const bool gram = METRIC != kAbsDiff;

  for (int item = blockIdx.x; item < g.n_items; item += gridDim.x) {
    const int rb = g.rb0 + item % g.n_rb;
    const int seg = item / g.n_rb;
    const int ct0 = seg * g.ct_per_item;
    const int ct1 = min(ct0 + g.ct_per_item, g.n_ct);
    const int row0 = rb * BM;
    __syncthreads();
    if (gram) load_tile_t(As, g.U, g.kp, row0);
    for (int i = threadIdx.x; i < BM; i += NT) Ap[i] = g.params[row0 + i];
    const float rmax_r = g.tile_rmax[rb];

    float rn[TM], rd[TM];
#pragma unroll
    for (int i = 0; i < TM; i++) rn[i] = rd[i] = 0.0f;

    for (int ct = ct0; ct < ct1; ct++) {
      const int col0 = ct * BM;
      __syncthreads();
      if (gram) load_tile_t(Bs, g.U, g.kp, col0);
      for (int i = threadIdx.x; i < BM; i += NT) Bp[i] = g.params[col0 + i];
      __syncthreads();

      float acc[TM][TM];
#pragma unroll
      for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TM; j++) acc[i][j] = 0.0f;
      if (gram) {
#pragma unroll 2
        for (int k = 0; k < g.kp; k++) {
          const float4 a0 = *reinterpret_cast<const float4*>(As + k * (BM + 4) + ty * TM);
          const float4 a1 = *reinterpret_cast<const float4*>(As + k * (BM + 4) + ty * TM + 4);
          const float4 b0 = *reinterpret_cast<const float4*>(Bs + k * (BM + 4) + tx * TM);
          const float4 b1 = *reinterpret_cast<const float4*>(Bs + k * (BM + 4) + tx * TM + 4);
          const float a[TM] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
          const float b[TM] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
          for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TM; j++) {
              if (diff_metric(METRIC)) {
                const float d = a[i] - b[j];
                acc[i][j] = fmaf(d, d, acc[i][j]);
              } else {
                acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
              }
            }
        }
      }
      const bool full = col0 + BM <= g.ec.n;
      const int cm = METRIC == kPearson ? c_mode(kEps * rmax_r * g.tile_rmax[ct]) : kCFirst;
      const bool diag = (ct == rb);
      if (full && !diag && cm == kCFirst)
        tile_epilogue<METRIC, kCFirst, true, false>(acc, Ap, Bp, row0, col0, g.ec, rn, rd);
      else if (full && !diag && cm == kCSecond)
        tile_epilogue<METRIC, kCSecond, true, false>(acc, Ap, Bp, row0, col0, g.ec, rn, rd);
      else if (cm == kCFirst)
        tile_epilogue<METRIC, kCFirst, false, true>(acc, Ap, Bp, row0, col0, g.ec, rn, rd);
      else if (cm == kCSecond)
        tile_epilogue<METRIC, kCSecond, false, true>(acc, Ap, Bp, row0, col0, g.ec, rn, rd);
      else
        tile_epilogue<METRIC, kCExact, false, true>(acc, Ap, Bp, row0, col0, g.ec, rn, rd);
    }
    // Reduce row partials over the 16 column-threads of each row group
    // (lanes tx = 0..15 of a half-warp), then one FP64 atomic per row.
#pragma unroll
    for (int i = 0; i < TM; i++) {
#pragma unroll
      for (int o = 8; o; o >>= 1) {
        rn[i] += __shfl_xor_sync(0xffffffffu, rn[i], o);
        rd[i] += __shfl_xor_sync(0xffffffffu, rd[i], o);
      }
    }
    if (tx == 0) {
#pragma unroll
      for (int i = 0; i < TM; i++) {
        const int r = row0 + ty * TM + i;
        if (r < g.ec.n) {
          atomicAdd(g.num + r, (double)rn[i]);
          atomicAdd(g.den + r, (double)rd[i]);
        }
      }
    }
  }
}

}  // namespace

cudaError_t launch_gram_fp32(const float* U, int kp, const BlockParams* params, const float* tile_rmax,
                             EpiConsts ec, double* num, double* den, int num_sms, cudaStream_t st, int rb_begin,
                             int rb_end) {
  Fp32Args g;
  g.U = U;
  g.kp = kp;
  g.params = params;
  g.tile_rmax = tile_rmax;
  g.ec = ec;
  g.num = num;
  g.den = den;
  g.n_ct = (ec.n + BM - 1) / BM;
  if (rb_end < 0) rb_end = g.n_ct;
  rb_end = std::min(rb_end, g.n_ct);
  if (rb_begin < 0 || rb_begin >= rb_end) return cudaSuccess;  // no rows in this range
  g.rb0 = rb_begin;
  g.n_rb = rb_end - rb_begin;
  // Split the column range so that there are at least ~4 items per SM.
  int segs = (4 * num_sms + g.n_rb - 1) / g.n_rb;
  if (segs > g.n_ct) segs = g.n_ct;
  if (segs < 1) segs = 1;
  g.ct_per_item = (g.n_ct + segs - 1) / segs;
  segs = (g.n_ct + g.ct_per_item - 1) / g.ct_per_item;
  g.n_items = g.n_rb * segs;
  size_t smem = (size_t)2 * kp * (BM + 4) * sizeof(float) + 2 * BM * sizeof(BlockParams);
  int grid = g.n_items < 2 * num_sms ? g.n_items : 2 * num_sms;
  cudaError_t e;
#define SRED_LAUNCH(M)                                                                           \
  e = cudaFuncSetAttribute(k_gram_fp32<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
  if (e != cudaSuccess) return e;                                                                \
  k_gram_fp32<M><<<grid, NT, smem, st>>>(g);
  switch (ec.metric) {
    case kPearson: SRED_LAUNCH(kPearson); break;
    case kSsim: SRED_LAUNCH(kSsim); break;
    case kNrmse: SRED_LAUNCH(kNrmse); break;
    case kNrmseW: SRED_LAUNCH(kNrmseW); break;
    case kNrmseD: SRED_LAUNCH(kNrmseD); break;
    case kNrmseDW: SRED_LAUNCH(kNrmseDW); break;
    case kDebugDot: SRED_LAUNCH(kDebugDot); break;
    default: SRED_LAUNCH(kAbsDiff); break;
  }
#undef SRED_LAUNCH
  return cudaGetLastError();
}

}  // namespace sred
