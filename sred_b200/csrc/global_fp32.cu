// Plain FP32 CUDA-core engine of the global repetition map.
//
// All-pairs Gram G = U U^T over the compacted relevant blocks (unit vectors,
// FP32), register-blocked 8x8 per thread on a 128x128 tile, with the fused
// per-pair epilogue (epilogue.cuh): the N x N similarity matrix is never
// stored.
//
// Same symmetric schedule as the tensor-core engine: only tiles of the upper
// triangle (row block rb <= column tile ct) are evaluated, pairs below the
// diagonal of the diagonal tiles are masked, and each pair's terms go to both
// blocks (the self pair once). A work item is (column tile ct, a run of up to L
// row blocks); the column tile and its parameters stay in shared memory for
// the item and its column sums in registers (8 columns per thread), while the
// row blocks stream through. Row sums leave once per tile (a butterfly over
// the 16 threads that share rows, then one FP64 atomic add per row), column
// sums once per item.
//
// This is the comparison form for the tensor-core engine: the same moments,
// compaction, schedule and epilogue, with FFMA contraction. For NRMSE it
// accumulates |u_p - u_q|^2 instead (diff_metric), the form without
// cancellation for near-identical blocks.
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
  int n_rb;              // 128-blocks holding valid rows (= column tiles)
  int L;                 // row blocks per item
  long long item0, item1;
};

__host__ __device__ inline long long items_before_fp32(long long ct, int L) {
  // sum over column tiles c < ct of ceil((c + 1) / L)
  const long long Q = ct / L, R = ct - Q * L;
  return (long long)L * Q * (Q + 1) / 2 + R * (Q + 1);
}

__device__ __forceinline__ void decode_item_fp32(long long it, const Fp32Args& g, int& ct, int& rb0, int& rb1) {
  int lo = 0, hi = g.n_rb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items_before_fp32(mid, g.L) <= it) lo = mid;
    else hi = mid - 1;
  }
  ct = lo;
  rb0 = (int)(it - items_before_fp32(lo, g.L)) * g.L;
  rb1 = min(rb0 + g.L, lo + 1);
}

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

// Pair terms of this thread's 8 x 8 pairs into the row sums rn/rd (per tile)
// and the column sums cn/cd (per item). MASKED: the diagonal or ragged tile
// (q >= p for the rows, q > p for the columns, both below n).
template <int METRIC, int CMODE, bool MASKED>
__device__ __forceinline__ void tile_epilogue(const float (&acc)[TM][TM], const BlockParams* __restrict__ rowp,
                                              const BlockParams* __restrict__ colp, int row0, int col0,
                                              const EpiConsts& ec, float (&rn)[TM], float (&rd)[TM],
                                              float (&cn)[TM], float (&cd)[TM]) {
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
#pragma unroll
  for (int i = 0; i < TM; i++) {
    const RowState rs = make_row(rowp[ty * TM + i], ec);
    const int p = row0 + ty * TM + i;
#pragma unroll
    for (int j = 0; j < TM; j++) {
      const int q = col0 + tx * TM + j;
      float G = acc[i][j];
      if (!diff_metric(METRIC) && MASKED && q == p && rs.r > 0.0f) G = 1.0f;
      float tn, td;
      pair_terms<METRIC, CMODE>(G, rs, colp[tx * TM + j], ec, tn, td);
      if (!MASKED) {
        rn[i] += tn;
        rd[i] += td;
        cn[j] += tn;
        cd[j] += td;
      } else {
        const bool rv = p < ec.n && q >= p && q < ec.n, cv = rv && q != p;
        rn[i] += rv ? tn : 0.0f;
        rd[i] += rv ? td : 0.0f;
        cn[j] += cv ? tn : 0.0f;
        cd[j] += cv ? td : 0.0f;
      }
    }
  }
}

// Sums of 16 values over the 16 lanes that share them (lanes with equal
// lane >> 4): stages xor 1, 2, 4, 8 each keep half the values; lane l ends with
// the full sum of value index (bit3 = l&1, bit2 = (l>>1)&1, bit1 = (l>>2)&1, bit0 = (l>>3)&1).
__device__ __forceinline__ float reduce16(const float (&x)[16], int& idx) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float y8[8], y4[4], y2[2];
  const bool b0 = lane & 1, b1 = lane & 2, b2 = lane & 4, b3 = lane & 8;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const float keep = b0 ? x[8 + i] : x[i], send = b0 ? x[i] : x[8 + i];
    y8[i] = keep + __shfl_xor_sync(full, send, 1);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float keep = b1 ? y8[4 + i] : y8[i], send = b1 ? y8[i] : y8[4 + i];
    y4[i] = keep + __shfl_xor_sync(full, send, 2);
  }
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const float keep = b2 ? y4[2 + i] : y4[i], send = b2 ? y4[i] : y4[2 + i];
    y2[i] = keep + __shfl_xor_sync(full, send, 4);
  }
  const float keep = b3 ? y2[1] : y2[0], send = b3 ? y2[0] : y2[1];
  idx = 8 * (int)b0 + 4 * (int)b1 + 2 * (int)b2 + (int)b3;
  return keep + __shfl_xor_sync(full, send, 8);
}

template <int METRIC>
__global__ void __launch_bounds__(NT, 2) k_gram_fp32(Fp32Args g) {
  extern __shared__ __align__(16) float smem[];
  float* As = smem;                                  // [kp][BM+4] rows (streamed)
  float* Bs = As + (size_t)g.kp * (BM + 4);          // [kp][BM+4] columns (held per item)
  BlockParams* Ap = reinterpret_cast<BlockParams*>(Bs + (size_t)g.kp * (BM + 4));  // [BM]
  BlockParams* Bp = Ap + BM;                                                         // [BM]
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  const bool gram = METRIC != kAbsDiff;

  for (long long it = g.item0 + blockIdx.x; it < g.item1; it += gridDim.x) {
    int ct, rb0, rb1;
    decode_item_fp32(it, g, ct, rb0, rb1);
    const int col0 = ct * BM;
    __syncthreads();
    if (gram) load_tile_t(Bs, g.U, g.kp, col0);
    for (int i = threadIdx.x; i < BM; i += NT) Bp[i] = g.params[col0 + i];
    const float rmax_c = g.tile_rmax[ct];
    const bool full = col0 + BM <= g.ec.n;
    float cn[TM], cd[TM];
#pragma unroll
    for (int j = 0; j < TM; j++) cn[j] = cd[j] = 0.0f;

    for (int rb = rb0; rb < rb1; rb++) {
      const int row0 = rb * BM;
      __syncthreads();
      if (gram) load_tile_t(As, g.U, g.kp, row0);
      for (int i = threadIdx.x; i < BM; i += NT) Ap[i] = g.params[row0 + i];
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
      const int cm = METRIC == kPearson ? c_mode(kEps * g.tile_rmax[rb] * rmax_c) : kCFirst;
      const bool masked = !full || rb == ct;
      float rn[TM], rd[TM];
#pragma unroll
      for (int i = 0; i < TM; i++) rn[i] = rd[i] = 0.0f;
      if (masked)
        tile_epilogue<METRIC, kCExact, true>(acc, Ap, Bp, row0, col0, g.ec, rn, rd, cn, cd);
      else if (cm == kCFirst)
        tile_epilogue<METRIC, kCFirst, false>(acc, Ap, Bp, row0, col0, g.ec, rn, rd, cn, cd);
      else if (cm == kCSecond)
        tile_epilogue<METRIC, kCSecond, false>(acc, Ap, Bp, row0, col0, g.ec, rn, rd, cn, cd);
      else
        tile_epilogue<METRIC, kCExact, false>(acc, Ap, Bp, row0, col0, g.ec, rn, rd, cn, cd);
      // Row sums of the 16 column-threads of each row group (a half-warp),
      // then one FP64 atomic per row and sum.
      float x[16];
#pragma unroll
      for (int i = 0; i < TM; i++) {
        x[2 * i] = rn[i];
        x[2 * i + 1] = rd[i];
      }
      int idx;
      const float s = reduce16(x, idx);
      const int r = row0 + ty * TM + (idx >> 1);
      if (r < g.ec.n) atomicAdd(((idx & 1) ? g.den : g.num) + r, (double)s);
    }
    // Column sums of the item: the two row groups of a warp (xor 16), then one
    // FP64 atomic per column, sum and warp.
    {
      const unsigned full_mask = 0xffffffffu;
      const bool hi = threadIdx.x & 16;
      float y[TM];
#pragma unroll
      for (int j = 0; j < TM; j++) {
        const float keep = hi ? cd[j] : cn[j], send = hi ? cn[j] : cd[j];
        y[j] = keep + __shfl_xor_sync(full_mask, send, 16);
      }
#pragma unroll
      for (int j = 0; j < TM; j++) {
        const int q = col0 + tx * TM + j;
        if (q < g.ec.n) atomicAdd((hi ? g.den : g.num) + q, (double)y[j]);
      }
    }
  }
}

}  // namespace

cudaError_t launch_gram_fp32(const float* U, int kp, const BlockParams* params, const float* tile_rmax,
                             EpiConsts ec, double* num, double* den, int num_sms, cudaStream_t st, int shard,
                             int n_shards) {
  if (n_shards < 1 || shard < 0 || shard >= n_shards) return cudaErrorInvalidValue;
  if (ec.n <= 0) return cudaSuccess;
  Fp32Args g;
  g.U = U;
  g.kp = kp;
  g.params = params;
  g.tile_rmax = tile_rmax;
  g.ec = ec;
  g.num = num;
  g.den = den;
  g.n_rb = (ec.n + BM - 1) / BM;
  // Items of up to 16 row blocks, fewer when that leaves under ~4 per SM slot.
  int L = 16;
  while (L > 1 && items_before_fp32(g.n_rb, L) < 8LL * num_sms) L >>= 1;
  g.L = L;
  const long long items = items_before_fp32(g.n_rb, L);
  g.item0 = items * shard / n_shards;
  g.item1 = items * (shard + 1) / n_shards;
  if (g.item0 >= g.item1) return cudaSuccess;
  size_t smem = (size_t)2 * kp * (BM + 4) * sizeof(float) + 2 * BM * sizeof(BlockParams);
  const int grid = (int)std::min<long long>(g.item1 - g.item0, 2LL * num_sms);
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
