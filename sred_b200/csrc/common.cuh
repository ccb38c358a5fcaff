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
              kHu = 6, kPhase = 7 /* block-map shape metrics */ };

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

// Epilogue constants shared by all tiles of one map.
struct EpiConsts {
  int metric;
  int n;            // valid blocks (rows == cols)
  float nrmse_scale;  // (K-1)/K
  float c1, c2;
};

// Launch the FP32 CUDA-core all-pairs kernel (global_fp32.cu).
// U: n_pad x kp floats (unit vectors), params: n_pad entries, num/den: n doubles (zeroed).
// Rows are processed in 128-row blocks; [rb_begin, rb_end) restricts the launch
// to those row blocks (rb_end < 0: all), the unit of row sharding.
cudaError_t launch_gram_fp32(const float* U, int kp, const BlockParams* params, const float* tile_rmax,
                             EpiConsts ec, double* num, double* den, int num_sms, cudaStream_t st,
                             int rb_begin = 0, int rb_end = -1);

// Column parameters of one 256-column tile, structure of arrays, as the
// tensor-core engine copies them into shared memory:
//   [a x256 | r x256 | sigma x256 | mu x256 | max r of the tile | 3 x pad]
constexpr int kColSoaFloats = 4 * 256 + 4;

// Launch the split-BF16 tcgen05 all-pairs kernel (global_tc.cu).
// A, B: n_pad x kq bf16 ([hi|lo|hi] and [hi|hi|lo]); colsoa: n_pad/256 tiles
// of kColSoaFloats (k_col_soa).
cudaError_t launch_gram_tc(const __nv_bfloat16* A, const __nv_bfloat16* B, int kq, int n_pad,
                           const BlockParams* params, const float* colsoa, const float* tile_rmax, EpiConsts ec,
                           double* num, double* den, int num_sms, int* status, cudaStream_t st,
                           int rb_begin = 0, int rb_end = -1);

}  // namespace sred
