// Shared definitions of libsred's device code and host orchestration.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/sred.h"

namespace sred {

constexpr float kEps = 0.0000001f;  // java/Utils.java:20 (Utils.EPSILON)
constexpr float kC1 = 0.0001f;      // cl/kernelGetGlobalSsim2D.cl:102
constexpr float kC2 = 0.0009f;      // cl/kernelGetGlobalSsim2D.cl:104
constexpr int kMaxK = 512;          // largest ellipse block size accepted

enum Metric { kPearson = 0, kSsim = 1, kNrmse = 2, kAbsDiff = 3, kCosine = 4,
              kDebugDot = 5 /* diagnostics: num += G a_p a_q, den += r_p + r_q */,
              kHu = 6, kPhase = 7 /* block-map shape metrics */,
              kNrmseW = 8 /* NRMSE with each term weighted (the 3D global kernel) */,
              // NRMSE from the accumulated squared difference of the unit
              // vectors (FP32 engine): unweighted (2D) and weighted (3D)
              kNrmseD = 9, kNrmseDW = 10,
              kHu7 = 11 /* block map: distance of the seven Hu invariants */ };

// The FP32 engine's accumulator holds sum_i (u_p,i - u_q,i)^2 instead of the
// dot product for these metrics.
__host__ __device__ constexpr bool diff_metric(int m) { return m == kNrmseD || m == kNrmseDW; }

// Ellipse pixel offsets (dx, dy), row-major ellipse order, as the kernels gather them.
struct Ellipse {
  int k;
  int rw, rh;
  short dx[kMaxK];
  short dy[kMaxK];
};

// Host: build the ellipse (java/GlobalRepetition2D_.java:102-111).
int build_ellipse(int bw, int bh, Ellipse* e);

// ---------------------------------------------------------------------------
// Per-block data of the global map, produced by the moment pass.
//   gram list: relevant, non-flat blocks (enter the all-pairs contraction)
//   flat list: relevant blocks with sigma == 0 (handled in closed form)
// ---------------------------------------------------------------------------
struct BlockParams {
  float a;      // sigma64 * sqrt(log2(e) / (noise_var + eps)): weight = 2^-(a_p - a_q)^2
  float e;      // eps / sigma64 (0 if sigma64 == 0)
  float r;      // 1 / sigma64 (0 if sigma64 == 0)
  float sigma;  // sigma64
  float mu;     // mu64
  float pad0, pad1, pad2;
};

// Split-BF16 operands of the tensor-core engine, u = hi + mid (+ lo), each
// part the BF16 rounding of what the previous parts leave of u:
//   two levels:   A = [hi|mid|hi], B = [hi|hi|mid] (3K columns); the products
//                 carry about 16 significand bits (dot-product error up to
//                 ~1e-5 for unit vectors);
//   three levels: A = [hi|mid|lo|hi|mid|hi], B = [hi|hi|hi|mid|mid|lo] (6K
//                 columns); every product down to 2^-18 relative, an FP32-level
//                 dot product. Used while 6K fits in 128 columns, where the
//                 tiles are bound by the epilogue and the deeper MMA is free,
//                 and always for NRMSE, whose 1 - G term needs it.
inline int split_levels(int K) { return 6 * K <= 128 ? 3 : 2; }
inline int split_cols(int K) { return split_levels(K) == 3 ? (6 * K + 31) / 32 * 32 : (3 * K + 31) / 32 * 32; }
inline bool nrmse_metric(int m) { return m == 2 /* kNrmse */ || m == 8 /* kNrmseW */; }
inline int split_levels_for(int metric, int K) { return nrmse_metric(metric) ? 3 : split_levels(K); }
inline int split_cols_for(int metric, int K) {
  return split_levels_for(metric, K) == 3 ? (6 * K + 31) / 32 * 32 : (3 * K + 31) / 32 * 32;
}

__device__ __forceinline__ void store_split(__nv_bfloat16* a, __nv_bfloat16* b, int K, int i, double u,
                                            int levels) {
  const __nv_bfloat16 hi = __float2bfloat16_rn((float)u);
  const double r = u - (double)__bfloat162float(hi);
  const __nv_bfloat16 mid = __float2bfloat16_rn((float)r);
  if (levels == 2) {
    a[i] = hi; a[K + i] = mid; a[2 * K + i] = hi;
    b[i] = hi; b[K + i] = hi; b[2 * K + i] = mid;
    return;
  }
  const __nv_bfloat16 lo = __float2bfloat16_rn((float)(r - (double)__bfloat162float(mid)));
  a[i] = hi; a[K + i] = mid; a[2 * K + i] = lo; a[3 * K + i] = hi; a[4 * K + i] = mid; a[5 * K + i] = hi;
  b[i] = hi; b[K + i] = hi; b[2 * K + i] = hi; b[3 * K + i] = mid; b[4 * K + i] = mid; b[5 * K + i] = lo;
}

// a / b, correctly rounded, for many a and one b: y = RN(1/b) once, then
// q = RN(a y), the exact residual r = a - b q (one FMA) and RN(q + r y).
// Markstein's theorem (P. Markstein, IBM J. Res. Dev. 34(1):111-119, 1990)
// makes the result the correctly rounded quotient when y is the correctly
// rounded reciprocal and q is within one ulp, barring underflow; tested
// against IEEE division (sred_debug_divide_fixed).
__device__ __forceinline__ float div_fixed(float a, float b, float y) {
  const float q = __fmul_rn(a, y);
  const float r = __fmaf_rn(-q, b, a);
  return __fmaf_rn(r, y, q);
}
// The same in FP64 (y = RN(1/b) from __drcp_rn); tested against IEEE
// division (sred_debug_divide_fixed64).
__device__ __forceinline__ double div_fixed(double a, double b, double y) {
  const double q = __dmul_rn(a, y);
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, y, q);
}

// Epilogue constants shared by all tiles of one map.
struct EpiConsts {
  int metric;
  int n;            // valid blocks (rows == cols)
  float nrmse_scale;  // (K-1)/K
  float c1, c2;
  // NRMSE on the tensor cores: pairs with G above nrmse_near get the term of
  // the exact squared difference of their FP32 unit vectors U (row pitch kp,
  // K values), the form the FP32 engine evaluates for every pair.
  const float* U = nullptr;
  int kp = 0, K = 0;
  float nrmse_near = 1.0f;
};

// Near-identical pairs (G > 1 - 2^-7) of tensor-core NRMSE take the exact
// difference form: there 1 - G is within an order of magnitude of the FP32
// accumulation error of G, which the square root of the term amplifies.
constexpr float kNrmseNear = 1.0f - 1.0f / 128.0f;

// Launch the FP32 CUDA-core all-pairs kernel (global_fp32.cu), on the same
// symmetric schedule as the tensor-core engine with 128 x 128 tiles.
// U: n_pad x kp floats (unit vectors), params: n_pad entries, num/den: n
// doubles (zeroed). The work items are split into n_shards equal ranges; this
// launch runs range `shard`.
cudaError_t launch_gram_fp32(const float* U, int kp, const BlockParams* params, const float* tile_rmax,
                             EpiConsts ec, double* num, double* den, int num_sms, cudaStream_t st,
                             int shard = 0, int n_shards = 1);

// Column parameters of one BN-column tile as the tensor-core engine copies
// them into shared memory: [a x BN | r x BN | sigma x BN | mu x BN | max r of
// the tile | 3 x pad], each array permuted within every 16-column group so that
// an epilogue thread's four columns of the group (2j, 2j + 1, 8 + 2j, 9 + 2j for
// j = t % 4) are one float4.
__host__ __device__ constexpr int col_soa_floats(int bn) { return 4 * bn + 4; }
__host__ __device__ constexpr int col_soa_pos(int i) {
  return (i & ~15) + 4 * ((i & 7) >> 1) + 2 * ((i >> 3) & 1) + (i & 1);
}
// Row parameters of one 128-row block: per row the pairs (a, a, -eps r, -eps r,
// sigma, sigma, mu, mu) as the epilogue's f32x2 operands, then r x 128, then
// max r and 3 x pad.
constexpr int kRowSoaFloats = 8 * 128 + 128 + 4;

// Launch shape of the tensor-core engine for a K': column tile width (256 or
// 128), whole-tile A buffers or a ring of 64-column chunks, dynamic shared
// memory. False if the B tile does not fit in shared memory.
struct TcPlan {
  int bn;
  bool tr;
  int stages;
  size_t smem;
};
bool plan_gram_tc(int kq, TcPlan* plan);

// Test hooks of the tensor-core engine: a wait limit (0: 4 s) and a tile whose
// operand copies the producer never issues (-1: none), so that the pipeline
// waits run out with nothing in flight.
struct TcDebug {
  unsigned long long timeout_ns;
  long long withhold_tile;
};

// A launch shape of the tensor-core engine (bn 0: the default plan): column
// tile width, whole-tile A buffers (tr 1) or the chunk ring (tr 0), and the
// largest run of row blocks per work item (L; the item-count rule may lower it).
struct TcChoice {
  int bn = 0, tr = 0, L = 0;
};
// The launch shapes that fit in shared memory for a K' (at most cap).
int gram_tc_candidates(int kq, TcChoice* out, int cap);

// Floats of the parameter workspace launch_gram_tc fills (column tiles and
// row blocks) for n_pad blocks.
size_t gram_tc_soa_floats(int n_pad);

// Work items of the symmetric schedule for n blocks and tile width bn (the
// upper triangle of 128-row x bn-column tiles in runs of L row blocks).
long long gram_tc_items(int n, int bn, int* L, int num_sms, int max_L = 0);

// Launch the split-BF16 tcgen05 all-pairs kernel (global_tc.cu).
// A, B: n_pad x kq bf16 (store_split); params: n_pad entries (rows past n
// zero); soa_ws: gram_tc_soa_floats(n_pad) floats of workspace; num/den: n
// doubles (zeroed), to which every pair's terms are added for both blocks.
// The upper-triangle work items are split into n_shards equal ranges; this
// launch runs range `shard` (the shards' num/den add up to the whole map).
cudaError_t launch_gram_tc(const __nv_bfloat16* A, const __nv_bfloat16* B, int kq, int n_pad,
                           const BlockParams* params, float* soa_ws, EpiConsts ec, double* num, double* den,
                           int num_sms, int* status, cudaStream_t st, int shard = 0, int n_shards = 1,
                           const TcDebug* dbg = nullptr, const TcChoice* choice = nullptr);

}  // namespace sred
